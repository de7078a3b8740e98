// clb_u1.cuh - sm_100a kernels of the complex scalar + U(1) gauge sector (lphi4U1).
//
// Restates, in the reference's rounding order (every product and sum pinned with the _rn
// intrinsics, so the FP64 path rounds where the reference's expression templates round):
//   ComplexScalarKernels::get   evolvers/kernels/complexscalarkernels.h:28-35
//   covLaplacianCS, U1 links    definitions/gaugederivatives.h:48-53, 92-102
//   U1Kernels::get              evolvers/kernels/u1kernels.h:31-52
//   U1Current, U1ChargeDensity  definitions/mattercurrents.h:27-76
//   grad2CS, B2U1, pi2U1        definitions/fieldfunctionals.h:80-153
//   GaussLaws::checkU1          definitions/gausslaws.h:34-53
//   ScaleFactorKernels::get     evolvers/kernels/scalefactorkernels.h:27-80 (complex scalar and U(1) terms)
//   Energies (CS, U(1))         definitions/energies.h:47-97, 217-239
//   lphi4U1 potential           models/lphi4U1.h:117-129 (V = c4 |phi|^4, dV/d|phi| = 4 c4 |phi|^3)
//
// Layout: ten FP64 arrays of N^3 sites (x slowest, z fastest), fields then momenta, components
// Re phi, Im phi, A_x, A_y, A_z.  Links U_i(x) = exp(-i dx gQ A_i(x)) are formed on the fly.

#pragma once

#include "clb_internal.cuh"

#include <type_traits>

namespace clb {

constexpr int kU1Red = 7;   // kick-sweep partial slots (see k_u1_kick)
constexpr int kU1Meas = 24; // measurement partial slots (see k_u1_measure)

// Scale factor, cached volume averages (the reference's CSpi2AvI, U1pi2AvI, ... of abstractmodel.h)
// and the per-sweep coefficients derived from them.
struct U1State {
  double aI, aSI, aIM, aDotI, aDotSI, aDotSIM;
  double csPi2I, csPi2SI, csPi2SIM, csGrad2I;
  double u1Pi2I, u1Pi2SI, u1Pi2SIM, u1Mag2I;
  double potI, potSI;
  double csGrad2SI, u1Mag2SI; // position Verlet: field averages at the half step (positionverlet.h:258-266)
  double cs_drift; // pow(aSI, alpha - 3)        (velocityverlet.h:195); position Verlet pow(aI, ...)
  double u1_drift; // pow(aSI, alpha - 1)        (velocityverlet.h:207)
  double kA;       // pow(aI, 1 + alpha)         (complexscalarkernels.h:33, u1kernels.h:45)
  double kB2;      // pow(aI, 3 + alpha) / 2     (complexscalarkernels.h:34)
  double kG;       // pow(aI, -1 + alpha)        (u1kernels.h:46)
  int32_t status, pad;
};

struct U1Params {
  int N;
  size_t n3;
  double dx, dx2, inv_dx2;
  double ndxg;  // (-dx) gQ: link phase per unit A
  double gQ, c4;
  double J0;    // 2/dx (fStar/omegaStar)^2            (mattercurrents.h:29, 70)
  double el0;   // 0.5 (omegaStar/fStar)^2             (energies.h:70, 80)
  double alpha, fm2, dt, inv_n3;
  int order; // site order of the kick and adjoint sweeps (for_sites)
};

// Kick factors of up to two successive kicks with the same kernel: complex scalar (dt/2 w, or
// w dt on the leapfrog) and U(1) (dt w / 2) (velocityverlet.h:141-157, leapfrog.h:141-155).
struct U1Kick {
  double hc[2], hu[2];
};

__device__ __forceinline__ double u1_m(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double u1_a(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double u1_s(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double u1_d(double a, double b) { return __ddiv_rn(a, b); }
// FP32 form: plain single-precision arithmetic (contraction allowed; a division by dx, dx^2 or
// |phi| is a multiply by the reciprocal)
__device__ __forceinline__ float u1_m(float a, float b) { return a * b; }
__device__ __forceinline__ float u1_a(float a, float b) { return a + b; }
__device__ __forceinline__ float u1_s(float a, float b) { return a - b; }
__device__ __forceinline__ float u1_d(float a, float b) { return a * (1.0f / b); } // reciprocal formed once per site
__device__ __forceinline__ void u1_sincos(double x, double *sn, double *cs) { sincos(x, sn, cs); }
__device__ __forceinline__ void u1_sincos(float x, float *sn, float *cs) { sincosf(x, sn, cs); }

// FP64 arithmetic of the adjoint's segment recompute, which is not bound to the reference's
// rounding order: products and sums may contract into FMAs, and a division becomes a multiply by
// the divisor's reciprocal (formed once per site for the lattice spacing).
struct FD {
  double v;
  FD() = default;
  __host__ __device__ constexpr FD(double x) : v(x) {}
  __host__ __device__ explicit constexpr operator double() const { return v; }
};
__device__ __forceinline__ FD u1_m(FD a, FD b) { return FD(a.v * b.v); }
__device__ __forceinline__ FD u1_a(FD a, FD b) { return FD(a.v + b.v); }
__device__ __forceinline__ FD u1_s(FD a, FD b) { return FD(a.v - b.v); }
__device__ __forceinline__ FD u1_d(FD a, FD b) { return FD(a.v * (1.0 / b.v)); }
__device__ __forceinline__ FD operator-(FD a) { return FD(-a.v); }
__device__ __forceinline__ FD sqrt(FD a) { return FD(::sqrt(a.v)); }
__device__ __forceinline__ void u1_sincos(FD x, FD *sn, FD *cs) { sincos(x.v, &sn->v, &cs->v); }

// Per-site kernel values in arithmetic type T.  Fields f (storage S): [Re phi, Im phi, A_x, A_y,
// A_z] x n3.  The FP64 form (S = T = double) pins every rounding; the FP32 form computes in float.
template <class T> struct U1Site {
  T fr, fi;            // phi(x)
  T wr[3], wi[3];      // U_i(x) phi(x + i)
  T g0[3][3];          // forwDiff(A_j, i)(x) = (A_j(x + i) - A_j(x)) / dx, [i][j]
  T Kr, Ki;            // complex scalar kernel
  T KA[3];             // U(1) kernel per direction
  T nrm;               // |phi|
};

template <bool KERNEL, class S, class T>
__device__ __forceinline__ void u1_site(const S *__restrict__ f, const U1Params &a, size_t s,
                                        const long long (&op)[3], const long long (&om)[3], T kA, T kB2, T kG,
                                        U1Site<T> &o)
{
  const size_t n3 = a.n3;
  const S *phr = f, *phi = f + n3;
  const S *A[3] = {f + 2 * n3, f + 3 * n3, f + 4 * n3};
  const T ndxg = (T)a.ndxg, dx = (T)a.dx, dx2 = (T)a.dx2, inv_dx2 = (T)a.inv_dx2, c4 = (T)a.c4;
  const T J0 = (T)a.J0, gQ = (T)a.gQ;
  o.fr = (T)phr[s];
  o.fi = (T)phi[s];
  T pr = 0, pim = 0, mr = 0, mim = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const size_t sp = s + op[d];
    T ur, ui;
    u1_sincos(u1_m(ndxg, (T)A[d][s]), &ui, &ur);
    const T gr = (T)phr[sp], gi = (T)phi[sp];
    o.wr[d] = u1_s(u1_m(ur, gr), u1_m(ui, gi));
    o.wi[d] = u1_a(u1_m(ur, gi), u1_m(ui, gr));
    if (KERNEL) {
      // conj(U_d(x - d)) phi(x - d)
      const size_t sm = s + om[d];
      T vr, vi;
      u1_sincos(u1_m(ndxg, (T)A[d][sm]), &vi, &vr);
      const T nvi = -vi, hr = (T)phr[sm], hi = (T)phi[sm];
      const T cr = u1_s(u1_m(vr, hr), u1_m(nvi, hi));
      const T ci = u1_a(u1_m(vr, hi), u1_m(nvi, hr));
      if (d == 0) {
        pr = o.wr[0];
        pim = o.wi[0];
        mr = cr;
        mim = ci;
      } else {
        pr = u1_a(pr, o.wr[d]);
        pim = u1_a(pim, o.wi[d]);
        mr = u1_a(mr, cr);
        mim = u1_a(mim, ci);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) o.g0[i][j] = u1_d(u1_s((T)A[j][s + op[i]], (T)A[j][s]), dx);
  o.nrm = sqrt(u1_a(u1_m(o.fr, o.fr), u1_m(o.fi, o.fi)));
  if (!KERNEL) return;
  // complex scalar: a^{1+alpha} covLap(phi) - a^{3+alpha}/2 (dV/d|phi|)/|phi| phi
  const T clr = u1_d(u1_s(u1_a(pr, mr), u1_m(T(6.0), o.fr)), dx2);
  const T cli = u1_d(u1_s(u1_a(pim, mim), u1_m(T(6.0), o.fi)), dx2);
  const T nd = u1_m(c4, u1_m(T(4.0), u1_m(u1_m(o.nrm, o.nrm), o.nrm)));
  const T q = u1_d(nd, o.nrm);
  o.Kr = u1_s(u1_m(kA, clr), u1_m(kB2, u1_m(q, o.fr)));
  o.Ki = u1_s(u1_m(kA, cli), u1_m(kB2, u1_m(q, o.fi)));
  // U(1): a^{alpha-1} (lapl A_i - sum_j backDiff_j forwDiff_i A_j) - a^{1+alpha} J_i
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T c = (T)A[i][s];
    T t[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) t[d] = u1_s(u1_a((T)A[i][s + op[d]], (T)A[i][s + om[d]]), u1_m(T(2.0), c));
    const T lap = u1_m(inv_dx2, u1_a(u1_a(t[0], t[1]), t[2]));
    T grad = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const size_t sj = s + om[j];
      const size_t sij = i == j ? s : s + op[i] + om[j]; // x + i - j
      const T g1 = u1_d(u1_s((T)A[j][sij], (T)A[j][sj]), dx);
      const T tj = u1_d(u1_s(o.g0[i][j], g1), dx);
      grad = j == 0 ? tj : u1_a(grad, tj);
    }
    const T im = u1_s(u1_m(o.wr[i], o.fi), u1_m(o.wi[i], o.fr));
    const T J = u1_m(J0, u1_m(gQ, im));
    o.KA[i] = u1_s(u1_m(kG, u1_s(lap, grad)), u1_m(kA, J));
  }
}

// sum_j |D+_j phi|^2 (fieldfunctionals.h:80-84) from the site's covariant neighbours
template <class T> __device__ __forceinline__ T u1_cs_grad2(const U1Site<T> &o, T dx)
{
  T acc = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const T dr = u1_d(u1_s(o.wr[j], o.fr), dx), di = u1_d(u1_s(o.wi[j], o.fi), dx);
    const T n2 = u1_a(u1_m(dr, dr), u1_m(di, di));
    acc = j == 0 ? n2 : u1_a(acc, n2);
  }
  return acc;
}

// F_21^2 + (F_31^2 + F_32^2), F_ij = forwDiff(A_j, i) - forwDiff(A_i, j) (fieldfunctionals.h:133-141)
template <class T> __device__ __forceinline__ T u1_b2(const U1Site<T> &o)
{
  const T f21 = u1_s(o.g0[1][0], o.g0[0][1]);
  const T f31 = u1_s(o.g0[2][0], o.g0[0][2]);
  const T f32 = u1_s(o.g0[2][1], o.g0[1][2]);
  return u1_a(u1_m(f21, f21), u1_a(u1_m(f31, f31), u1_m(f32, f32)));
}

template <class T> __device__ __forceinline__ T u1_pot(const U1Site<T> &o, T c4)
{
  return u1_m(c4, u1_m(u1_m(u1_m(o.nrm, o.nrm), o.nrm), o.nrm));
}

// Kick sweep: NK (0, 1 or 2) successive in-place kicks of all five momenta with the kernel at the
// current fields.  Partials per block: [0,1] complex-scalar |pi|^2 and U(1) sum pi_i^2 after the
// first kick (or of the momenta as they are, NK = 0), [2] sum |D phi|^2, [3] B^2, [4] V, [5,6] the
// momentum sums after the second kick.  RF adds the field slots, RP the momentum slots.
// Two resident 256-thread blocks per SM (128 registers): the sweep is latency-bound, and the
// doubled occupancy outweighs the few spills (1.65x over one block at 128^3).
#ifndef CLB_U1_KICK_MINB
#define CLB_U1_KICK_MINB 2
#endif
// SAVE (adjoint recompute): also writes the fields and the momenta after the first kick, the state
// at the stage boundary between the two kicks, to save_f / save_p.  FAST (FP64 storage only):
// the kernel values in FD arithmetic.
template <int NK, bool RF, bool RP, class S, bool SAVE = false, bool FAST = false>
__global__ void __launch_bounds__(256, CLB_U1_KICK_MINB)
    k_u1_kick(const S *__restrict__ f, S *__restrict__ p, U1Params a, U1Kick kc, const U1State *__restrict__ st,
              double *__restrict__ partials, S *__restrict__ save_f = nullptr, S *__restrict__ save_p = nullptr)
{
  __shared__ double smem[(256 / 32) * kU1Red];
  using T = typename std::conditional<FAST && sizeof(S) == 8, FD, S>::type;
  const size_t n3 = a.n3;
  const T kA = (T)st->kA, kB2 = (T)st->kB2, kG = (T)st->kG;
  double acc[kU1Red];
#pragma unroll
  for (int k = 0; k < kU1Red; ++k) acc[k] = 0;
  for_sites(a.N, n3, a.order, [&](size_t s) {
    long long op[3], om[3];
    u1_offsets(a.N, s, op, om);
    U1Site<T> o;
    u1_site<(NK > 0)>(f, a, s, op, om, kA, kB2, kG, o);
    if (RF) {
      acc[2] += (double)u1_cs_grad2(o, (T)a.dx);
      acc[3] += (double)u1_b2(o);
      acc[4] += (double)u1_pot(o, (T)a.c4);
    }
    // momenta and their increments in FP64 (FP32 storage: rounded once per kick)
    double q[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) q[c] = (double)p[c * n3 + s];
#pragma unroll
    for (int k = 0; k < (NK > 0 ? NK : 1); ++k) {
      if (NK > 0) {
        q[0] = u1_a(q[0], u1_m(kc.hc[k], (double)o.Kr));
        q[1] = u1_a(q[1], u1_m(kc.hc[k], (double)o.Ki));
#pragma unroll
        for (int i = 0; i < 3; ++i) q[2 + i] = u1_a(q[2 + i], u1_m(kc.hu[k], (double)o.KA[i]));
        if (sizeof(S) == 4) {
#pragma unroll
          for (int c = 0; c < 5; ++c) q[c] = (double)(S)q[c]; // the stored value after this kick
        }
        if (SAVE && k == 0) {
#pragma unroll
          for (int c = 0; c < 5; ++c) {
            save_p[c * n3 + s] = (S)q[c];
            save_f[c * n3 + s] = f[c * n3 + s];
          }
        }
      }
      if (RP) {
        acc[k == 0 ? 0 : 5] += u1_a(u1_m(q[0], q[0]), u1_m(q[1], q[1]));
        acc[k == 0 ? 1 : 6] += u1_a(u1_a(u1_m(q[2], q[2]), u1_m(q[3], q[3])), u1_m(q[4], q[4]));
      }
    }
    if (NK > 0) {
#pragma unroll
      for (int c = 0; c < 5; ++c) p[c * n3 + s] = (S)q[c];
    }
  });
  if (RF || RP) {
    block_reduce<kU1Red, 256>(acc, smem);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < kU1Red; ++k) partials[(size_t)blockIdx.x * kU1Red + k] = acc[k];
    }
  }
}

// ---- the kick on staged planes ----------------------------------------------------------------
// One block per (z, y) tile of BZ x BY sites (one per thread) and an x-run of LX planes; the
// blocks take tiles in turn (grid-stride over tiles, so the partial rows are the grid's).  Each
// x-plane of the five field components, with a one-cell halo in y and z (corners included: the
// curl term reads x + i - j), is copied by cp.async into a ring of D shared-memory slots, D - 3
// planes ahead of the plane being kicked, whose x - 1 and x + 1 neighbours stay in the ring.  The
// site arithmetic is u1_site's, on a view of the ring: the component stride is the ring's and the
// neighbour offsets are ring offsets, so every site's kernel values are bitwise those of
// k_u1_kick; only the order of the volume sums differs.
template <class S> struct U1Ring {
  static constexpr int BZ = 32, BY = 8, THREADS = BZ * BY;
  static constexpr int ROW = BZ + 2, PLANE = (BY + 2) * ROW; // one component's plane with halos
  static constexpr int D = sizeof(S) == 8 ? 6 : 8;           // ring slots
  static constexpr int CS = D * PLANE;                       // component stride in the ring
  static constexpr int BYTES = 5 * CS * (int)sizeof(S);
};

// SAVE and FAST as in k_u1_kick (the adjoint's segment recompute).
template <int NK, bool RF, bool RP, class S, bool SAVE = false, bool FAST = false>
__global__ void __launch_bounds__(256, CLB_U1_KICK_MINB)
    k_u1_kick_tile(const S *__restrict__ f, S *__restrict__ p, U1Params a, U1Kick kc, const U1State *__restrict__ st,
                   double *__restrict__ partials, int LX, S *__restrict__ save_f = nullptr,
                   S *__restrict__ save_p = nullptr)
{
  using RG = U1Ring<S>;
  constexpr int BZ = RG::BZ, BY = RG::BY, ROW = RG::ROW, PL = RG::PLANE, D = RG::D, L = D - 2;
  static_assert(L >= 2, "two planes ahead at least");
  extern __shared__ __align__(16) unsigned char u1_ring_raw[];
  S *const ring = reinterpret_cast<S *>(u1_ring_raw); // [5][D][BY + 2][ROW]
  __shared__ double smem[(256 / 32) * kU1Red];
  using T = typename std::conditional<FAST && sizeof(S) == 8, FD, S>::type;
  const int N = a.N;
  const size_t n3 = a.n3;
  U1Params av = a;
  av.n3 = (size_t)RG::CS; // u1_site reads component c of ring index t at ring[c * CS + t]
  const T kA = (T)st->kA, kB2 = (T)st->kB2, kG = (T)st->kG;
  const int tz = threadIdx.x % BZ, ty = threadIdx.x / BZ;
  const int gz = (N + BZ - 1) / BZ, gy = (N + BY - 1) / BY, gxr = (N + LX - 1) / LX;
  const long long ntiles = (long long)gz * gy * gxr;
  auto wrap = [&](int v) { return v < 0 ? v + N : (v >= N ? v - N : v); };
  double acc[kU1Red];
#pragma unroll
  for (int k = 0; k < kU1Red; ++k) acc[k] = 0;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int z0 = (int)(tile % gz) * BZ, y0 = (int)((tile / gz) % gy) * BY, x0 = (int)(tile / ((long long)gz * gy)) * LX;
    const int x1 = min(N, x0 + LX), hz = min(BZ, N - z0), hy = min(BY, N - y0);
    const bool valid = tz < hz && ty < hy;
    // plane j of the run (x = x0 - 1 + j, up to x1) into slot j % D: the (hy + 2) x (hz + 2) box
    auto issue = [&](int j) {
      const int xp = x0 - 1 + j;
      if (xp <= x1) {
        const size_t xs = (size_t)wrap(xp);
        S *slot = ring + (j % D) * PL;
        for (int cell = threadIdx.x; cell < PL; cell += RG::THREADS) {
          const int r = cell / ROW, c = cell - r * ROW;
          if (r > hy + 1 || c > hz + 1) continue;
          const size_t g = (xs * N + (size_t)wrap(y0 - 1 + r)) * N + (size_t)wrap(z0 - 1 + c);
#pragma unroll
          for (int comp = 0; comp < 5; ++comp) cp_async<(int)sizeof(S)>(slot + comp * RG::CS + cell, f + comp * n3 + g);
        }
      }
      cp_async_commit(); // one group per plane, empty past the run
    };
#pragma unroll 1
    for (int j = 0; j <= L; ++j) issue(j);
#pragma unroll 1
    for (int x = x0; x < x1; ++x) {
      const int j = x - x0 + 1;
      cp_async_wait<L - 2>(); // planes up to x + 1 have landed (this thread's copies)
      __syncthreads();        // ... and every thread's; slot (j + L) % D, plane x - 2's, is free
      issue(j + L);
      if (valid) {
        const int sc = j % D, sp = (j + 1) % D, sm = (j - 1) % D;
        const size_t t = (size_t)sc * PL + (size_t)(ty + 1) * ROW + (size_t)(tz + 1);
        const long long op[3] = {(long long)(sp - sc) * PL, ROW, 1};
        const long long om[3] = {(long long)(sm - sc) * PL, -ROW, -1};
        U1Site<T> o;
        u1_site<(NK > 0)>(ring, av, t, op, om, kA, kB2, kG, o);
        if (RF) {
          acc[2] += (double)u1_cs_grad2(o, (T)a.dx);
          acc[3] += (double)u1_b2(o);
          acc[4] += (double)u1_pot(o, (T)a.c4);
        }
        const size_t g = ((size_t)x * N + (size_t)(y0 + ty)) * N + (size_t)(z0 + tz);
        double q[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) q[c] = (double)p[c * n3 + g];
#pragma unroll
        for (int k = 0; k < (NK > 0 ? NK : 1); ++k) {
          if (NK > 0) {
            q[0] = u1_a(q[0], u1_m(kc.hc[k], (double)o.Kr));
            q[1] = u1_a(q[1], u1_m(kc.hc[k], (double)o.Ki));
#pragma unroll
            for (int i = 0; i < 3; ++i) q[2 + i] = u1_a(q[2 + i], u1_m(kc.hu[k], (double)o.KA[i]));
            if (sizeof(S) == 4) {
#pragma unroll
              for (int c = 0; c < 5; ++c) q[c] = (double)(S)q[c]; // the stored value after this kick
            }
            if (SAVE && k == 0) {
#pragma unroll
              for (int c = 0; c < 5; ++c) {
                save_p[c * n3 + g] = (S)q[c];
                save_f[c * n3 + g] = ring[c * RG::CS + t];
              }
            }
          }
          if (RP) {
            acc[k == 0 ? 0 : 5] += u1_a(u1_m(q[0], q[0]), u1_m(q[1], q[1]));
            acc[k == 0 ? 1 : 6] += u1_a(u1_a(u1_m(q[2], q[2]), u1_m(q[3], q[3])), u1_m(q[4], q[4]));
          }
        }
        if (NK > 0) {
#pragma unroll
          for (int c = 0; c < 5; ++c) p[c * n3 + g] = (S)q[c];
        }
      }
    }
    cp_async_wait<0>(); // only empty groups remain past the run
    __syncthreads();    // the next tile refills the ring
  }
  if (RF || RP) {
    block_reduce<kU1Red, 256>(acc, smem);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < kU1Red; ++k) partials[(size_t)blockIdx.x * kU1Red + k] = acc[k];
    }
  }
}

// Drifts phi += ((pow(aSI, alpha-3) dt) w) pi_phi and A += ((pow(aSI, alpha-1) w) dt) pi_A
// (velocityverlet.h:193-210; the leapfrog's forms leapfrog.h:203-217 are w = 1).
template <class S>
__global__ void __launch_bounds__(256)
    k_u1_drift(S *__restrict__ f, const S *__restrict__ p, size_t n3, double w, double dt,
               const U1State *__restrict__ st)
{
  const double cc = u1_m(u1_m(st->cs_drift, dt), w);
  const double cu = u1_m(u1_m(st->u1_drift, w), dt);
  const size_t n = 5 * n3, n2 = 2 * n3;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    f[i] = (S)u1_a((double)f[i], u1_m(i < n2 ? cc : cu, (double)p[i]));
}

// ScaleFactorKernels::get with complex-scalar and U(1) energies (scalefactorkernels.h:73-77,
// energies.h:47-97).
__device__ __forceinline__ double u1_sf_kernel(const U1State &s, const U1Params &p)
{
  const double al = p.alpha;
  const double e4 = u1_m(p.el0, ipow_d(s.aI, -4));
  const double Ekcs = u1_m(s.csPi2I, ipow_d(s.aI, -6));
  const double Egcs = u1_m(s.csGrad2I, ipow_d(s.aI, -2));
  const double Eel = u1_m(e4, s.u1Pi2I), Emag = u1_m(e4, s.u1Mag2I);
  const double br = u1_a(u1_a(u1_a(u1_m(al - 2, Ekcs), u1_m(al, Egcs)), u1_m(al - 1, u1_a(Eel, Emag))),
                         u1_m(al + 1, s.potI));
  return u1_m(u1_m(pow(s.aI, 2 * al + 1) / 3.0, p.fm2), br);
}


// ScaleFactorKernels::getSI with complex-scalar and U(1) energies (scalefactorkernels.h:83-119):
// the half-step averages at aI.
__device__ __forceinline__ double u1_sf_kernel_si(const U1State &s, const U1Params &p)
{
  const double al = p.alpha;
  const double e4 = u1_m(p.el0, ipow_d(s.aI, -4));
  const double Ekcs = u1_m(s.csPi2SI, ipow_d(s.aI, -6));
  const double Egcs = u1_m(s.csGrad2SI, ipow_d(s.aI, -2));
  const double Eel = u1_m(e4, s.u1Pi2SI), Emag = u1_m(e4, s.u1Mag2SI);
  const double br = u1_a(u1_a(u1_a(u1_m(al - 2, Ekcs), u1_m(al, Egcs)), u1_m(al - 1, u1_a(Eel, Emag))),
                         u1_m(al + 1, s.potSI));
  return u1_m(u1_m(pow(s.aI, 2 * al + 1) / 3.0, p.fm2), br);
}

// One-thread tail: fixed-order sum of the kick-sweep partials and the scale-factor update, in
// the order of the VelocityVerlet and LeapFrog schedules (same flags as the scalar tail).
// Fixed-order sum of the kick-sweep partial rows (all threads of one 256-thread block; the
// totals are valid in thread 0).
__device__ __forceinline__ void u1_reduce_partials(const double *__restrict__ partials, int nblocks,
                                                   double (&v)[kU1Red], double *smem)
{
#pragma unroll
  for (int k = 0; k < kU1Red; ++k) v[k] = 0;
  if (nblocks <= 0) return;
#pragma unroll 5
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < kU1Red; ++k) v[k] += partials[(size_t)b * kU1Red + k];
  }
  block_reduce<kU1Red, 256>(v, smem);
}

// The scale-factor update of one tail on the state s from the reduced sums v.
__device__ __forceinline__ void u1_tail_apply(U1State &s, const double (&v)[kU1Red], const TailOp &op, const U1Params &p)
{
  const double csP = v[0] * p.inv_n3, u1P = v[1] * p.inv_n3, csG = v[2] * p.inv_n3, u1B = v[3] * p.inv_n3;
  const double pot = v[4] * p.inv_n3, csP2 = v[5] * p.inv_n3, u1P2 = v[6] * p.inv_n3;
  const double dt = p.dt;
  const uint32_t fl = op.flags;
  if (fl & T_STORE_ALL) { // Averages::setAllAverages (averages.h:349-378)
    s.potI = s.potSI = pot;
    s.u1Pi2I = s.u1Pi2SI = u1P;
    s.u1Mag2I = u1B;
    s.csPi2I = s.csPi2SI = csP;
    s.csGrad2I = csG;
  }
  auto write_hist = [&]() {
    double *r = op.hist + op.hist_row * kHistCols;
    r[0] = s.aI;
    r[1] = s.aDotI;
    r[2] = s.csPi2I;
    r[3] = s.csGrad2I;
    r[4] = s.potI;
  };
  const bool hist = op.hist != nullptr && op.hist_row >= 0;
  if (fl & T_STORE_FIELDS) {
    s.csGrad2I = csG;
    s.u1Mag2I = u1B;
    s.potI = pot;
  }
  if (hist && (fl & T_HIST_EARLY)) write_hist();
  if (fl & T_STORE_PI2_I) {
    s.csPi2I = csP;
    s.u1Pi2I = u1P;
  }
  if (fl & T_STORE_PI2_LF) { // leapfrog.h:152-167
    s.csPi2SIM = s.csPi2SI;
    s.csPi2SI = csP;
    s.csPi2I = 0.5 * (s.csPi2SIM + s.csPi2SI);
    s.u1Pi2SIM = s.u1Pi2SI;
    s.u1Pi2SI = u1P;
    s.u1Pi2I = 0.5 * (s.u1Pi2SIM + s.u1Pi2SI);
  }
  if (fl & T_CORRECT_ADOT) { // HubbleConstraint::get RHS with Energies::rho (energies.h:217-239)
    const double e4 = u1_m(p.el0, ipow_d(s.aI, -4));
    const double rho = u1_a(u1_a(u1_a(u1_a(u1_m(s.csPi2I, ipow_d(s.aI, -6)), u1_m(s.csGrad2I, ipow_d(s.aI, -2))),
                                      u1_m(e4, s.u1Pi2I)),
                                 u1_m(e4, s.u1Mag2I)),
                            s.potI);
    s.aDotI = sqrt(u1_m(u1_m(pow(s.aI, 2 * p.alpha + 2) / 3., p.fm2), rho));
  }
  if (fl & T_VV_KICK_ONE) s.aDotI = u1_a(s.aDotSI, u1_m(u1_m(dt / 2, u1_sf_kernel(s, p)), op.w));
  if (hist && !(fl & T_HIST_EARLY)) write_hist();
  if (fl & T_LF_SYNC) s.aDotI = u1_a(s.aDotSI, u1_m(dt / 2.0, u1_sf_kernel(s, p)));
  if (fl & T_LF_CTOR) s.aDotSI = u1_s(s.aDotI, u1_m(dt / 2.0, u1_sf_kernel(s, p)));
  if (fl & T_LF_KICK) {
    s.aDotSIM = s.aDotSI;
    s.aDotSI = u1_a(s.aDotSI, u1_m(dt, u1_sf_kernel(s, p)));
    s.aDotI = (s.aDotSIM + s.aDotSI) / 2.0;
  }
  if (fl & T_LF_DRIFT) {
    s.aIM = s.aI;
    s.aI = u1_a(s.aI, u1_m(dt, s.aDotSI));
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  if (fl & T_VV_KICK_HALF) s.aDotSI = u1_a(s.aDotI, u1_m(u1_m(dt / 2, u1_sf_kernel(s, p)), op.w2));
  if (fl & T_STORE_PI2_B) {
    s.csPi2I = csP2;
    s.u1Pi2I = u1P2;
  }
  if (fl & T_VV_DRIFT) {
    s.aIM = s.aI;
    s.aI = u1_a(s.aI, u1_m(u1_m(dt, s.aDotSI), op.w2));
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  // PositionVerlet (positionverlet.h:160-163, 207-276), as in the scalar tail
  if (fl & T_PV_STORE_SI) {
    s.csGrad2SI = csG;
    s.u1Mag2SI = u1B;
    s.potSI = pot;
  }
  if (fl & T_PV_STORE_PI2) {
    s.csPi2SIM = s.csPi2I; // CSpi2AvIM
    s.u1Pi2SIM = s.u1Pi2I;
    s.csPi2I = csP;
    s.u1Pi2I = u1P;
    s.csPi2SI = 0.5 * (s.csPi2I + s.csPi2SIM);
    s.u1Pi2SI = 0.5 * (s.u1Pi2I + s.u1Pi2SIM);
  }
  if (fl & T_PV_KICK) s.aDotI = u1_a(s.aDotI, u1_m(u1_m(dt, u1_sf_kernel_si(s, p)), op.w));
  if (fl & T_PV_DRIFT_A2) {
    s.aI = u1_a(s.aI, u1_m(u1_m(dt / 2.0, s.aDotI), op.w));
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  if (fl & T_PV_DRIFT_A1) {
    s.aIM = s.aI;
    s.aI = u1_a(s.aI, u1_m(u1_m(dt / 2.0, s.aDotI), op.w2));
    s.aSI = s.aI;
  }
  // fixed background: the host's closed-form values (fixedbackgroundexpansion.h:37-45)
  if (fl & T_FB_AIM) s.aIM = s.aI;
  if (fl & T_FB_AI) s.aI = op.fa;
  if (fl & T_FB_ASI) s.aSI = op.fb;
  if (fl & T_FB_PV_HALF) {
    s.aIM = s.aI;
    s.aI = op.fb;
    s.aSI = s.aI;
  }
  if (fl & T_FB_ADOT) s.aDotI = op.fb;
  const double ad = (fl & T_PV_MODE) ? ((fl & (T_PV_DRIFT_A1 | T_FB_PV_HALF)) ? s.aIM : s.aI) : s.aSI;
  s.cs_drift = pow(ad, p.alpha - 3);
  s.u1_drift = pow(ad, p.alpha - 1);
  s.kA = pow(s.aI, 1 + p.alpha);
  s.kB2 = pow(s.aI, 3 + p.alpha) / 2;
  s.kG = pow(s.aI, -1 + p.alpha);
  if (!isfinite(s.aI) || !isfinite(s.aDotI) || !isfinite(s.aDotSI) || !isfinite(s.csPi2I) || !isfinite(s.u1Pi2I) ||
      !isfinite(s.csGrad2I) || !isfinite(s.u1Mag2I) || !isfinite(s.potI))
    s.status = 1;
}

static __global__ void __launch_bounds__(256)
    k_u1_tail(const double *__restrict__ partials, TailOp op, U1State *__restrict__ st, U1Params p)
{
  __shared__ double smem[(256 / 32) * kU1Red];
  double v[kU1Red];
  u1_reduce_partials(partials, op.nblocks, v, smem);
  if (threadIdx.x != 0) return;
  U1State s = *st;
  u1_tail_apply(s, v, op, p);
  *st = s;
}

// A stage boundary of the adjoint's segment recompute in one launch: the tail of the merged
// sweep's first kick (a), the boundary's record row, then the tail of its second kick (b, if
// b.flags), both from one reduction of the partials; the same values as k_u1_tail(a),
// k_u1_record, k_u1_tail(b).
static __global__ void __launch_bounds__(256)
    k_u1_tail_split(const double *__restrict__ partials, TailOp a, TailOp b, U1State *__restrict__ st, U1Params p,
                    U1State *__restrict__ rec, int64_t row)
{
  __shared__ double smem[(256 / 32) * kU1Red];
  double v[kU1Red];
  u1_reduce_partials(partials, a.nblocks, v, smem);
  if (threadIdx.x != 0) return;
  U1State s = *st;
  u1_tail_apply(s, v, a, p);
  rec[row] = s;
  if (b.flags) u1_tail_apply(s, v, b, p);
  *st = s;
}

// Measurement sums (one sweep): [0] |pi_phi|^2, [1] sum |D phi|^2, [2] sum pi_A^2, [3] B^2, [4] V,
// [5..10] Re phi, (Re phi)^2, Im phi, (Im phi)^2, |phi|, |phi|^2, [11..16] the same of pi_phi,
// [17] |pi_A|, [18] |B|, [19..22] Gauss |LHS - RHS|, |sum of squares|, |RHS|, |LHS|
// (gausslaws.h:34-53 with U1ChargeDensity, mattercurrents.h:27-48).
// FP32 storage is measured in FP64 arithmetic on the stored values.
template <class S>
__global__ void __launch_bounds__(256)
    k_u1_measure(const S *__restrict__ f, const S *__restrict__ p, U1Params a, double *__restrict__ partials)
{
  __shared__ double smem[(256 / 32) * kU1Meas];
  const size_t n3 = a.n3;
  double acc[kU1Meas];
#pragma unroll
  for (int k = 0; k < kU1Meas; ++k) acc[k] = 0;
  const double gnorm = u1_m(a.J0, a.gQ);
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    long long op[3], om[3];
    u1_offsets(a.N, s, op, om);
    U1Site<double> o;
    u1_site<false>(f, a, s, op, om, 0.0, 0.0, 0.0, o);
    const double pr = (double)p[s], pi = (double)p[n3 + s];
    double q[3], l[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      q[i] = (double)p[(2 + i) * n3 + s];
      l[i] = u1_s(q[i], (double)p[(2 + i) * n3 + s + om[i]]);
    }
    const double cp2 = u1_a(u1_m(pr, pr), u1_m(pi, pi));
    const double up2 = u1_a(u1_a(u1_m(q[0], q[0]), u1_m(q[1], q[1])), u1_m(q[2], q[2]));
    const double b2 = u1_b2(o);
    acc[0] += cp2;
    acc[1] += u1_cs_grad2(o, a.dx);
    acc[2] += up2;
    acc[3] += b2;
    acc[4] += u1_pot(o, a.c4);
    acc[5] += o.fr;
    acc[6] += u1_m(o.fr, o.fr);
    acc[7] += o.fi;
    acc[8] += u1_m(o.fi, o.fi);
    acc[9] += o.nrm;
    acc[10] += u1_m(o.nrm, o.nrm);
    const double pn = sqrt(cp2);
    acc[11] += pr;
    acc[12] += u1_m(pr, pr);
    acc[13] += pi;
    acc[14] += u1_m(pi, pi);
    acc[15] += pn;
    acc[16] += u1_m(pn, pn);
    acc[17] += sqrt(up2);
    // |B| with B_1 = F_32, B_2 = F_13, B_3 = F_21
    {
      const double b1 = u1_s(o.g0[2][1], o.g0[1][2]), bb = u1_s(o.g0[0][2], o.g0[2][0]), b3 = u1_s(o.g0[1][0], o.g0[0][1]);
      acc[18] += sqrt(u1_a(u1_a(u1_m(b1, b1), u1_m(bb, bb)), u1_m(b3, b3)));
    }
    // Gauss: LHS = sum_i (pi_i(x) - pi_i(x - i)) / dx, RHS = -dx rho, rho = (J0 gQ) Im(conj(pi_phi) phi)
    const double LHS = u1_d(u1_a(u1_a(l[0], l[1]), l[2]), a.dx);
    const double im = u1_s(u1_m(pr, o.fi), u1_m(pi, o.fr));
    const double RHS = u1_m(-a.dx, u1_m(gnorm, im));
    const double L1 = u1_d(l[0], a.dx), L2 = u1_d(l[1], a.dx), L3 = u1_d(l[2], a.dx);
    const double diff = u1_s(LHS, RHS);
    const double sum = u1_a(u1_a(u1_a(u1_m(L1, L1), u1_m(L2, L2)), u1_m(L3, L3)), u1_m(RHS, RHS));
    acc[19] += fabs(diff);
    acc[20] += fabs(sum);
    acc[21] += fabs(RHS);
    acc[22] += fabs(LHS);
  }
  block_reduce<kU1Meas, 256>(acc, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kU1Meas; ++k) partials[(size_t)blockIdx.x * kU1Meas + k] = acc[k];
  }
}

} // namespace clb
