// clb_adjoint.cuh - reverse-mode (adjoint) sweeps of the lphi4U1 velocity-Verlet stage.
//
// The forward map of one VV stage with weight w (velocityverlet.h:51-114, 140-210) is
//   1  aDotS = aDot0 + dt/2 w F(a0, <.>(q0, p0))
//   2  p1 = p0 + h K(q0; a0)                       h = dt/2 w (scalar), dt w / 2 (U(1))
//   3  a1 = a0 + dt w aDotS,  aS = (a0 + a1) / 2
//   4  q1 = q0 + dt w D(aS) p1                     D = aS^(alpha-3) (scalar), aS^(alpha-1) (U(1))
//   5  p2 = p1 + h K(q1; a1)
//   6  aDot1 = aDotS + dt/2 w F(a1, <.>(q1, p2))
// with q = (Re phi, Im phi, A_x, A_y, A_z), p the momenta and <.> the five volume averages
// <|pi_phi|^2>, <sum_i |D_i phi|^2>, <sum_i pi_i^2>, <B^2>, <V> that enter F
// (scalefactorkernels.h:73-77).
//
// The kernel is a metric gradient: K = -M^{-1} dU/dq with
//   U = a^{1+alpha} U_D + a^{3+alpha}/2 sum V + m_A a^{alpha-1} U_B,  M = diag(1, 1, m_A, m_A, m_A),
//   U_D = 1/(2 dx^2) sum |U_i phi(x+i) - phi(x)|^2,  U_B = 1/2 sum_{i<j} F_ij^2,  m_A = 1/(2 (fStar/omegaStar)^2),
// which reproduces complexscalarkernels.h:33-34 and u1kernels.h:44-50 term by term.  Its Jacobian
// J = dK/dq is therefore M^{-1}-symmetric and the transposed kick J^T lambda equals M J (M^{-1} lambda):
// a Jacobian-vector product, evaluated here with dual numbers over the same stencil.  The gradients
// of the averages are read off the same pieces: d<|D phi|^2>/dphi = -2/N^3 covLap,
// d<|D phi|^2>/dA_i = 1/N^3 (2 gQ/dx) Im(conj(U_i phi(x+i)) phi), d<B^2>/dA = -2/N^3 curl curl A,
// d<V>/dphi = 1/N^3 dV/dphi.
//
// The coupling gQ enters U only through U_D(phi, gQ A), so dU/dgQ = (1/gQ) sum_x,i A_i dU_D'/dA_i
// (U_D' = a^{1+alpha} U_D), and for any cotangent lt of the momenta
//   lt . dK/dgQ = (m_A/gQ) sum_x,i [A_i (J^D w)_i + w_i K^D_i],   w = M^{-1} lt,
// with K^D_i = -kA J0 gQ Im(conj(U_i phi(x+i)) phi) the U_D part of the U(1) kernel and J^D w its
// derivative along w: the one dual lane of the state direction also gives the coupling
// derivative.  Likewise d(sum |D phi|^2)/dgQ = (2/dx) sum A_i Im(conj(U_i phi(x+i)) phi).
//
// One sweep per stage boundary runs backwards.  It fuses the two transposed kicks that act on the
// fields there: part A, the first kick of the stage that starts at the boundary (maps 2 and 1 of
// that stage), and part B, the second kick of the stage that ends there (maps 6, 5 and 4).  Both
// kicks use the kernel at the same fields and scale factor, J^T is linear, and the momentum-average
// gradients between them are local to each site, so one JVP along
//   w = M^{-1} (hA . lambda_A + hB . lambda_B),  lambda_A = pbar,  lambda_B = pbar + (momentum-average terms)
// gives both.  The scalar steps (F, a, aDot) are formed on the host between sweeps from the per-site
// dot products the sweeps reduce.

#pragma once

#include "clb_internal.cuh"
#include "clb_tangent.cuh"
#include "clb_u1.cuh"

namespace clb {

using TD = Tan<double>;

__device__ __forceinline__ void sincos_t(TD t, TD &s, TD &c)
{
  double sv, cv;
  sincos(t.v, &sv, &cv);
  s = TD(sv, cv * t.d);
  c = TD(cv, -sv * t.d);
}

// Stencil pieces of the lphi4U1 kernel at one site, as values with their derivative along w.
struct U1Pieces {
  TD cl[2];     // covariant Laplacian of phi
  TD dv[2];     // dV/dphi_c = 4 c4 |phi|^2 phi_c
  TD cc[3];     // lapl A_i - sum_j backDiff_j forwDiff_i A_j
  TD im[3];     // Im(conj(U_i phi(x+i)) phi(x))
  double vn[2]; // |phi|^2 phi_c (d dV/dphi_c / d c4 / 4)
  double n4;    // |phi|^4 (dV / d c4)
};

// ld(c, site) returns component c at a site as (value, derivative along w).
template <class LD>
__device__ __forceinline__ void u1_pieces(LD ld, const U1Params &a, size_t s, const long long (&op)[3],
                                          const long long (&om)[3], U1Pieces &o)
{
  const double ndxg = -a.dx * a.gQ;
  const TD fr = ld(0, s), fi = ld(1, s);
  TD pr(0.0), pim(0.0), mr(0.0), mim(0.0);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const size_t sp = s + op[d], sm = s + om[d];
    TD ur, ui, vr, vi;
    sincos_t(ndxg * ld(2 + d, s), ui, ur);
    const TD gr = ld(0, sp), gi = ld(1, sp);
    const TD wr = ur * gr - ui * gi, wi = ur * gi + ui * gr;
    sincos_t(ndxg * ld(2 + d, sm), vi, vr);
    const TD hr = ld(0, sm), hi = ld(1, sm);
    pr = pr + wr;
    pim = pim + wi;
    mr = mr + (vr * hr + vi * hi);
    mim = mim + (vr * hi - vi * hr);
    o.im[d] = wr * fi - wi * fr;
  }
  o.cl[0] = (pr + mr - 6.0 * fr) * a.inv_dx2;
  o.cl[1] = (pim + mim - 6.0 * fi) * a.inv_dx2;
  const TD n2 = fr * fr + fi * fi;
  o.dv[0] = (4.0 * a.c4) * (n2 * fr);
  o.dv[1] = (4.0 * a.c4) * (n2 * fi);
  o.vn[0] = n2.v * fr.v;
  o.vn[1] = n2.v * fi.v;
  o.n4 = n2.v * n2.v;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const TD c = ld(2 + i, s);
    TD acc(0.0);
#pragma unroll
    for (int d = 0; d < 3; ++d) acc = acc + (ld(2 + i, s + op[d]) + ld(2 + i, s + om[d]) - 2.0 * c);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const size_t sij = i == j ? s : s + op[i] + om[j];
      acc = acc - ((ld(2 + j, s + op[i]) - ld(2 + j, s)) - (ld(2 + j, sij) - ld(2 + j, s + om[j])));
    }
    o.cc[i] = acc * a.inv_dx2;
  }
}

struct U1AdjArgs {
  double hA[2], hB[2];         // kick factors (phi, A) of part A and part B; 0: no such kick
  double ApiA, AEA, ApiB, AEB; // cotangents of <|pi_phi|^2>, <sum pi_A^2> at part A's and part B's map
  double AD, AB, AV;           // cotangents of <|D phi|^2>, <B^2>, <V>, both parts
  double cdf, cda;             // transposed drift of part B: dt w D(aS) per group (0: none)
  double kA, kB2, kG;          // kick coefficients at the boundary's a
  double dkA, dkB2, dkG;       // their a-derivatives
  double J0;                   // 2/dx (fStar/omegaStar)^2
  double r2;                   // 2 (fStar/omegaStar)^2 = 1/m_A
  double inv_n3;
};

// [0] a-derivative dot of part A, [1] of part B, [2] d/dgQ and [3] d/dc4 of both kicks, [4]
// d(sum |D phi|^2)/dgQ, [5] sum |phi|^4, [6] [7] part B's drift dots (phi, A)
constexpr int kAdjSlots = 8;

// S is the storage type of the forward state (f, p); the cotangents are FP64 in either form.
// Reads qbar and pbar_in (lambda_A); writes qbar and pbar_out = lambda_B + (transposed drift).
// Two resident 256-thread blocks per SM (128 registers): 1.30x over one block at 254 registers;
// three are slower (spills).
#ifndef CLB_U1_ADJ_MINB
#define CLB_U1_ADJ_MINB 2
#endif
template <class S>
__global__ void __launch_bounds__(256, CLB_U1_ADJ_MINB)
    k_u1_adj(const S *__restrict__ f, const S *__restrict__ p, const double *__restrict__ pbar_in,
             double *__restrict__ qbar, double *__restrict__ pbar_out, U1Params a, U1AdjArgs g,
             double *__restrict__ partials)
{
  __shared__ double smem[(256 / 32) * kAdjSlots];
  const size_t n3 = a.n3;
  double acc[kAdjSlots];
#pragma unroll
  for (int k = 0; k < kAdjSlots; ++k) acc[k] = 0;
  const double two_n3 = 2.0 * g.inv_n3;
  const double cP = (g.ApiA + g.ApiB) * two_n3, cE = (g.AEA + g.AEB) * two_n3;
  const double kJ = g.kA * g.J0 * a.gQ;
  // loop invariants; the adjoint is not bound to the forward's rounding order, so its divides
  // by dx^2 and by m_A^-1 are multiplies by reciprocals
  const double inv_r2 = 1.0 / g.r2, cJ = g.kA * g.J0 * inv_r2, cD = g.AD * g.inv_n3 * (2.0 * a.gQ / a.dx);
  const double two_dx = 2.0 / a.dx, dJ = g.dkA * g.J0 * a.gQ;
  for_sites(a.N, n3, a.order, [&](size_t s) {
    long long op[3], om[3];
    u1_offsets(a.N, s, op, om);
    // the JVP direction at a site: M^{-1} (hA lambda_A + hB lambda_B)
    auto ld = [&](int c, size_t y) -> TD {
      const double lA = pbar_in[c * n3 + y];
      const int sec = c < 2 ? 0 : 1;
      const double lB = lA + (sec == 0 ? cP : cE) * (double)p[c * n3 + y];
      const double w = g.hA[sec] * lA + g.hB[sec] * lB;
      return TD((double)f[c * n3 + y], sec == 0 ? w : g.r2 * w);
    };
    U1Pieces o;
    u1_pieces(ld, a, s, op, om, o);
    // kernel values and derivatives (complexscalarkernels.h:33-34, u1kernels.h:50)
    TD K[5];
    K[0] = g.kA * o.cl[0] - g.kB2 * o.dv[0];
    K[1] = g.kA * o.cl[1] - g.kB2 * o.dv[1];
#pragma unroll
    for (int i = 0; i < 3; ++i) K[2 + i] = g.kG * o.cc[i] - kJ * o.im[i];
    double lA[5], lB[5], qb[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      lA[c] = pbar_in[c * n3 + s];
      lB[c] = lA[c] + (c < 2 ? cP : cE) * (double)p[c * n3 + s];
      qb[c] = qbar[c * n3 + s];
    }
    // both transposed kicks: qbar += M J w
    qb[0] += K[0].d;
    qb[1] += K[1].d;
#pragma unroll
    for (int i = 0; i < 3; ++i) qb[2 + i] += K[2 + i].d * inv_r2;
    // gradients of the field averages
#pragma unroll
    for (int c = 0; c < 2; ++c) qb[c] += g.AD * (-two_n3) * o.cl[c].v + g.AV * g.inv_n3 * o.dv[c].v;
#pragma unroll
    for (int i = 0; i < 3; ++i)
      qb[2 + i] += cD * o.im[i].v + g.AB * (-two_n3) * o.cc[i].v;
    // scale-factor and coupling dot products
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double da = g.dkA * o.cl[c].v - g.dkB2 * o.dv[c].v;
      acc[0] += g.hA[0] * lA[c] * da;
      acc[1] += g.hB[0] * lB[c] * da;
      acc[3] += (g.hA[0] * lA[c] + g.hB[0] * lB[c]) * (-g.kB2 * 4.0 * o.vn[c]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double da = g.dkG * o.cc[i].v - dJ * o.im[i].v;
      acc[0] += g.hA[1] * lA[2 + i] * da;
      acc[1] += g.hB[1] * lB[2 + i] * da;
      const double Ai = (double)f[(2 + i) * n3 + s];
      const double wi = g.r2 * (g.hA[1] * lA[2 + i] + g.hB[1] * lB[2 + i]);
      acc[2] += -cJ * (Ai * o.im[i].d + wi * o.im[i].v);
      acc[4] += two_dx * Ai * o.im[i].v;
    }
    acc[5] += o.n4;
    // part B's transposed drift: pbar = lambda_B + dt w D qbar; its aS dot uses the momentum
    // before part B's kick, p - hB K
    double pb[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const bool phi = c < 2;
      const double p1 = (double)p[c * n3 + s] - g.hB[phi ? 0 : 1] * K[c].v;
      pb[c] = lB[c] + (phi ? g.cdf : g.cda) * qb[c];
      acc[phi ? 6 : 7] += p1 * qb[c];
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      qbar[c * n3 + s] = qb[c];
      pbar_out[c * n3 + s] = pb[c];
    }
  });
  block_reduce<kAdjSlots, 256>(acc, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kAdjSlots; ++k) partials[(size_t)blockIdx.x * kAdjSlots + k] = acc[k];
  }
}

// The same sweep on staged planes: each x-plane of the state (f, p) and of the incoming cotangent
// lambda_A, with a one-cell y/z halo (corners included), is copied by cp.async into a ring of D
// shared-memory slots ahead of use; the JVP direction at a cell is formed from the ring as k_u1_adj
// forms it from global memory, and u1_pieces runs on ring indices, so every site's values are
// those of k_u1_adj.  32 x 4-site tiles, one site per thread, two 128-thread blocks per SM (the
// registers of one 256-thread block: no spills); the blocks take tiles in turn, so the partial rows
// are the grid's.
template <class S> struct U1AdjRing {
  static constexpr int BZ = 32, BY = 4, THREADS = BZ * BY;
  static constexpr int ROW = BZ + 2, PLANE = (BY + 2) * ROW;
  static constexpr int D = 4, CS = D * PLANE;
  static constexpr int BYTES = 5 * CS * (2 * (int)sizeof(S) + (int)sizeof(double));
};

template <class S>
__global__ void __launch_bounds__(128, 2)
    k_u1_adj_tile(const S *__restrict__ f, const S *__restrict__ p, const double *__restrict__ pbar_in,
                  double *__restrict__ qbar, double *__restrict__ pbar_out, U1Params a, U1AdjArgs g,
                  double *__restrict__ partials, int LX)
{
  using RG = U1AdjRing<S>;
  constexpr int BZ = RG::BZ, BY = RG::BY, ROW = RG::ROW, PL = RG::PLANE, D = RG::D, CS = RG::CS, L = D - 2;
  extern __shared__ __align__(16) unsigned char adj_ring_raw[];
  double *const rL = reinterpret_cast<double *>(adj_ring_raw); // [5][D][BY + 2][ROW] lambda_A
  S *const rF = reinterpret_cast<S *>(rL + 5 * CS);             // fields
  S *const rP = rF + 5 * CS;                                   // momenta
  __shared__ double smem[(128 / 32) * kAdjSlots];
  const int N = a.N;
  const size_t n3 = a.n3;
  double acc[kAdjSlots];
#pragma unroll
  for (int k = 0; k < kAdjSlots; ++k) acc[k] = 0;
  const double two_n3 = 2.0 * g.inv_n3;
  const double cP = (g.ApiA + g.ApiB) * two_n3, cE = (g.AEA + g.AEB) * two_n3;
  const double kJ = g.kA * g.J0 * a.gQ;
  const double inv_r2 = 1.0 / g.r2, cJ = g.kA * g.J0 * inv_r2, cD = g.AD * g.inv_n3 * (2.0 * a.gQ / a.dx);
  const double two_dx = 2.0 / a.dx, dJ = g.dkA * g.J0 * a.gQ;
  const int tz = threadIdx.x % BZ, ty = threadIdx.x / BZ;
  const int gz = (N + BZ - 1) / BZ, gy = (N + BY - 1) / BY, gxr = (N + LX - 1) / LX;
  const long long ntiles = (long long)gz * gy * gxr;
  auto wrap = [&](int v) { return v < 0 ? v + N : (v >= N ? v - N : v); };
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int z0 = (int)(tile % gz) * BZ, y0 = (int)((tile / gz) % gy) * BY, x0 = (int)(tile / ((long long)gz * gy)) * LX;
    const int x1 = min(N, x0 + LX), hz = min(BZ, N - z0), hy = min(BY, N - y0);
    const bool valid = tz < hz && ty < hy;
    auto issue = [&](int j) {
      const int xp = x0 - 1 + j;
      if (xp <= x1) {
        const size_t xs = (size_t)wrap(xp);
        const int so = (j % D) * PL;
        for (int cell = threadIdx.x; cell < PL; cell += RG::THREADS) {
          const int r = cell / ROW, c = cell - r * ROW;
          if (r > hy + 1 || c > hz + 1) continue;
          const size_t y = (xs * N + (size_t)wrap(y0 - 1 + r)) * N + (size_t)wrap(z0 - 1 + c);
#pragma unroll
          for (int comp = 0; comp < 5; ++comp) {
            cp_async<(int)sizeof(S)>(rF + comp * CS + so + cell, f + comp * n3 + y);
            cp_async<(int)sizeof(S)>(rP + comp * CS + so + cell, p + comp * n3 + y);
            cp_async<8>(rL + comp * CS + so + cell, pbar_in + comp * n3 + y);
          }
        }
      }
      cp_async_commit();
    };
    // the JVP direction at ring index y: M^{-1} (hA lambda_A + hB lambda_B), as k_u1_adj's ld
    auto ld = [&](int c, size_t y) -> TD {
      const double lA = rL[c * CS + y];
      const int sec = c < 2 ? 0 : 1;
      const double lB = lA + (sec == 0 ? cP : cE) * (double)rP[c * CS + y];
      const double w = g.hA[sec] * lA + g.hB[sec] * lB;
      return TD((double)rF[c * CS + y], sec == 0 ? w : g.r2 * w);
    };
#pragma unroll 1
    for (int j = 0; j <= L; ++j) issue(j);
#pragma unroll 1
    for (int x = x0; x < x1; ++x) {
      const int j = x - x0 + 1;
      cp_async_wait<L - 2>();
      __syncthreads();
      issue(j + L);
      if (valid) {
        const int sc = j % D, sp = (j + 1) % D, sm = (j - 1) % D;
        const size_t t = (size_t)sc * PL + (size_t)(ty + 1) * ROW + (size_t)(tz + 1);
        const long long op[3] = {(long long)(sp - sc) * PL, ROW, 1};
        const long long om[3] = {(long long)(sm - sc) * PL, -ROW, -1};
        const size_t s = ((size_t)x * N + (size_t)(y0 + ty)) * N + (size_t)(z0 + tz);
        U1Pieces o;
        u1_pieces(ld, a, t, op, om, o);
        TD K[5];
        K[0] = g.kA * o.cl[0] - g.kB2 * o.dv[0];
        K[1] = g.kA * o.cl[1] - g.kB2 * o.dv[1];
#pragma unroll
        for (int i = 0; i < 3; ++i) K[2 + i] = g.kG * o.cc[i] - kJ * o.im[i];
        double lA[5], lB[5], qb[5], pc[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          lA[c] = rL[c * CS + t];
          pc[c] = (double)rP[c * CS + t];
          lB[c] = lA[c] + (c < 2 ? cP : cE) * pc[c];
          qb[c] = qbar[c * n3 + s];
        }
        qb[0] += K[0].d;
        qb[1] += K[1].d;
#pragma unroll
        for (int i = 0; i < 3; ++i) qb[2 + i] += K[2 + i].d * inv_r2;
#pragma unroll
        for (int c = 0; c < 2; ++c) qb[c] += g.AD * (-two_n3) * o.cl[c].v + g.AV * g.inv_n3 * o.dv[c].v;
#pragma unroll
        for (int i = 0; i < 3; ++i)
          qb[2 + i] += cD * o.im[i].v + g.AB * (-two_n3) * o.cc[i].v;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const double da = g.dkA * o.cl[c].v - g.dkB2 * o.dv[c].v;
          acc[0] += g.hA[0] * lA[c] * da;
          acc[1] += g.hB[0] * lB[c] * da;
          acc[3] += (g.hA[0] * lA[c] + g.hB[0] * lB[c]) * (-g.kB2 * 4.0 * o.vn[c]);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const double da = g.dkG * o.cc[i].v - dJ * o.im[i].v;
          acc[0] += g.hA[1] * lA[2 + i] * da;
          acc[1] += g.hB[1] * lB[2 + i] * da;
          const double Ai = (double)rF[(2 + i) * CS + t];
          const double wi = g.r2 * (g.hA[1] * lA[2 + i] + g.hB[1] * lB[2 + i]);
          acc[2] += -cJ * (Ai * o.im[i].d + wi * o.im[i].v);
          acc[4] += two_dx * Ai * o.im[i].v;
        }
        acc[5] += o.n4;
        double pb[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          const bool phi = c < 2;
          const double p1 = pc[c] - g.hB[phi ? 0 : 1] * K[c].v;
          pb[c] = lB[c] + (phi ? g.cdf : g.cda) * qb[c];
          acc[phi ? 6 : 7] += p1 * qb[c];
        }
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          qbar[c * n3 + s] = qb[c];
          pbar_out[c * n3 + s] = pb[c];
        }
      }
    }
    cp_async_wait<0>();
    __syncthreads();
  }
  block_reduce<kAdjSlots, 128>(acc, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kAdjSlots; ++k) partials[(size_t)blockIdx.x * kAdjSlots + k] = acc[k];
  }
}

// The cotangent of a momentum average <|pi_phi|^2> (or <sum pi_A^2>) with cotangent X adds
// 2 X / N^3 p to the momenta's cotangent: pbar += cphi p on the complex-scalar components and
// cA p on the gauge ones (set: pbar = that instead).  The leapfrog adjoint adds these after a
// boundary's sweep, once the scale-factor chain has given them.
template <class S>
__global__ void __launch_bounds__(256)
    k_u1_pbar_axpy(double *__restrict__ pbar, const S *__restrict__ p, size_t n3, double cphi, double cA, int set)
{
  const size_t n = 5 * n3, n2 = 2 * n3;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = (i < n2 ? cphi : cA) * (double)p[i];
    pbar[i] = set ? v : pbar[i] + v;
  }
}

// Copies the U(1) scalar state into row r of the per-boundary record (adjoint recompute).
__global__ void k_u1_record(const U1State *__restrict__ st, U1State *__restrict__ rec, int64_t r) { rec[r] = *st; }

} // namespace clb
