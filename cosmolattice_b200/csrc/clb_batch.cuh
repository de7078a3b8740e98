// clb_batch.cuh - sm_100a kernels of the batched lphi4 ensemble (many independent lattices).
//
// Every member is one real scalar singlet of the model header the library is built with (lphi4:
// V = c0/4 phi^4, models/lphi4.h:154-206 with the daughter field removed) on its own N^3 periodic
// lattice; the members share dt, evolver and expansion
// mode and differ in N, dx, c0, initial state and scale factor.  One launch of k_batch_sweep
// advances all members by one fused VV stage (the same drift + two-kick sweep as the single
// lattice path: velocityverlet.h:51-114, 129-196); k_batch_tail then updates each member's scale
// factor from its own fixed-order volume sums (scalefactorkernels.h:27-80).
//
// Storage: the members' N^3 arrays are concatenated (each starting on a 128-byte boundary).  FP64
// stores the fields themselves; FP32 stores each member's deviation from its FP64 homogeneous
// reference (DevState::ref_phi/ref_pi), as the single-lattice FP32/FP64-split form does.
#pragma once

#include "clb_internal.cuh"
#include "clb_scalar.cuh"
#include "clb_sweep.cuh"

#include <cooperative_groups.h>

namespace clb {

struct BatchLat {
  int N, gx, gy, gz, LX; // sweep grid of this member: (z, y) tiles of BZ x BY, x runs of LX planes
  int first_block, nblocks;
  long long off;         // element offset of the member's arrays
  double inv_dx2;
  ModelCouplings mc; // the member's couplings in the model header's form
  SFParams sp;
};

// VZ consecutive values to global memory (vector stores when VZ > 1; aligned: N % VZ == 0).
template <class R, int VZ> __device__ __forceinline__ void stg_v(R *p, const R (&v)[VZ])
{
  if constexpr (VZ == 1)
    p[0] = v[0];
  else
    stv<R, VZ>(p, v);
}

// The shared-memory ring of one tile: D slots, each one x-plane of fields and one of momenta,
// (BY + 2) rows (the y halos in rows 0 and BY + 1) of ROW elements: the z-left halo in column
// VZ - 1, the tile's sites from column VZ (aligned for VZ-wide copies), the z-right halo after
// them.  D: as many planes as fit in 32 KB, 3 to 8; the loads run D - 2 planes ahead of the plane
// whose x-neighbour is read.
template <int BZ, int BY, int VZ, class R> struct Ring {
  static constexpr int TZ = BZ * VZ;
  static constexpr int ROW = TZ + 2 * VZ;
  static constexpr int PLANE = (BY + 2) * ROW;
  static constexpr int PLANE_BYTES = 2 * PLANE * (int)sizeof(R);
  static constexpr int FIT = 32768 / PLANE_BYTES;
  static constexpr int D = FIT > 8 ? 8 : (FIT < 3 ? 3 : FIT);
  static constexpr int BYTES = D * PLANE_BYTES;
};

// DRIFT / KICK / RED as in k_sweep; one block = one (BZ VZ) x BY (z, y) tile of one member, each
// thread owning VZ consecutive z sites (every member's N a multiple of VZ), marching over LX
// x-planes.  Tile shape, VZ and LX are chosen by the batch autotuner.
// Each x-plane of the tile (with its y and z halos) is copied to a slot of the shared-memory ring
// (Ring) by cp.async, D - 2 planes ahead of use, so that several planes of loads are in flight
// per thread while one is computed.  The drift is applied where a value is read (a neighbour's
// drifted value is recomputed from its field and momentum: the same inputs give the same value).
// fin/pin are never written; fout/pout alias them only without DRIFT (the in-place kick writes
// only momenta of the block's own sites, which only this thread reads).
// Register budget: that of four resident 256-thread blocks per SM (64 registers) for one site per
// thread, twice that for vector sites.
#ifndef CLB_BATCH_MINB
#define CLB_BATCH_MINB 4
#endif

// One tile of one member: the member's block `local` of its (z, y, x-run) grid, with the block's
// sums of the averages in v (thread 0).  k_batch_sweep runs one tile per block; the persistent
// k_batch_persist runs a cluster's share of a member's tiles one after another.  The ring is the
// kernel's dynamic shared memory (Ring::BYTES).
template <int BZ, int BY, int VZ, class R, bool DRIFT, bool KICK, int RED>
__device__ __forceinline__ void batch_tile(const R *fin, const R *pin, R *fout, R *pout, const BatchLat &lt,
                                           DevState *__restrict__ st, int local, int rs, double dtw_d, double h1,
                                           double h2, double (&vout)[kRedSlots])
{
  using A = Ar<R>;
  using RG = Ring<BZ, BY, VZ, R>;
  constexpr bool SPLIT = sizeof(R) == 4;
  constexpr int TZ = RG::TZ, ROW = RG::ROW, PL = RG::PLANE, D = RG::D, L = D - 1;
  extern __shared__ __align__(16) unsigned char clb_batch_ring[];
  R *const ringF = reinterpret_cast<R *>(clb_batch_ring);
  R *const ringP = ringF + D * PL;
  __shared__ double red_smem[(BZ * BY / 32) * kRedSlots];
  const int bx = local % lt.gx, by = (local / lt.gx) % lt.gy, bz = local / (lt.gx * lt.gy);
  const int N = lt.N;
  fin += lt.off;
  pin += lt.off;
  fout += lt.off;
  pout += lt.off;
  const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * BZ + tz;
  const int z0 = bx * TZ, y0 = by * BY;
  const int hz = min(TZ, N - z0), hy = min(BY, N - y0);
  const int x0 = bz * lt.LX, x1 = min(N, x0 + lt.LX);
  const int zt = VZ * tz;                     // the thread's first z inside the tile
  const bool valid = zt < hz && ty < hy;      // then all VZ sites are inside (N % VZ == 0)
  const int y = y0 + ty, z = z0 + zt;
  const int ym = y0 == 0 ? N - 1 : y0 - 1, yp = y0 + hy == N ? 0 : y0 + hy;
  const int zm = z0 == 0 ? N - 1 : z0 - 1, zp = z0 + hz == N ? 0 : z0 + hz;

  // the member's reference step (split form) and its coefficients
  RefStep<1> rf{};
  ModelFluct spc{};
  if constexpr (SPLIT) {
    rf = ref_step<1>(st, rs, DRIFT, KICK, dtw_d, h1, h2, lt.mc);
    spc = ModelFluct::make(rf.phi[0], lt.mc);
    if ((DRIFT || KICK) && local == 0 && tid == 0) {
      st->ref_phi[rs ^ 1][0] = rf.phi[0];
      st->ref_pi[rs ^ 1][0] = rf.pi_next[0];
    }
  }
  const R pd = DRIFT ? (R)st->drift_p : R(0), dtw = DRIFT ? (R)dtw_d : R(0);
  const R KA = KICK ? (R)st->kick_A : R(0), KB = KICK ? (R)st->kick_B : R(0);
  const R inv_dx2 = (R)lt.inv_dx2, two = R(2);
  const float h1f = (float)h1, h2f = (float)h2;

  auto sidx = [&](int x, int yy, int zz) -> size_t { return ((size_t)x * N + yy) * N + zz; };
  auto wrapx = [&](int xx) { return xx >= N ? xx - N : (xx < 0 ? xx + N : xx); };
  constexpr bool LOADP = DRIFT || KICK || (RED & 1);
  const bool hym = ty == 0, hyp = ty == hy - 1, hzm = tz == 0, hzp = zt + VZ == hz;
  const int ctr = (ty + 1) * ROW + VZ + zt; // the thread's first site in a slot
  // Plane j of the tile's sequence (x = x0 - 1 + j) into slot j % D: the thread's own sites, and
  // for the computed planes x0 .. x1 - 1 the halo values it owns; momenta where they are read.
  auto issue = [&](int j) {
    const int xp = x0 - 1 + j;
    if (valid && xp <= x1) {
      const int xs = wrapx(xp);
      const bool halo = xp >= x0 && xp < x1;
      R *F = ringF + (j % D) * PL, *P = ringP + (j % D) * PL;
      const size_t s = sidx(xs, y, z);
      cp_run<R, VZ>(F + ctr, fin + s);
      if (LOADP) cp_run<R, VZ>(P + ctr, pin + s);
      if (halo) {
        if (hym) {
          cp_run<R, VZ>(F + VZ + zt, fin + sidx(xs, ym, z));
          if (DRIFT) cp_run<R, VZ>(P + VZ + zt, pin + sidx(xs, ym, z));
        }
        if (hyp) {
          cp_run<R, VZ>(F + (hy + 1) * ROW + VZ + zt, fin + sidx(xs, yp, z));
          if (DRIFT) cp_run<R, VZ>(P + (hy + 1) * ROW + VZ + zt, pin + sidx(xs, yp, z));
        }
        if (hzm) {
          cp_run<R, 1>(F + ctr - 1, fin + sidx(xs, y, zm));
          if (DRIFT) cp_run<R, 1>(P + ctr - 1, pin + sidx(xs, y, zm));
        }
        if (hzp) {
          cp_run<R, 1>(F + ctr + VZ, fin + sidx(xs, y, zp));
          if (DRIFT) cp_run<R, 1>(P + ctr + VZ, pin + sidx(xs, y, zp));
        }
      }
    }
    cp_async_commit(); // one group per plane, empty past the run
  };
  // the drifted field at element e of slot j
  auto fval = [&](int j, int e) -> R {
    const R f = ringF[(j % D) * PL + e];
    return DRIFT ? drift_val<R>(f, ringP[(j % D) * PL + e], pd, dtw) : f;
  };

  double acc_pi2 = 0, acc_g2 = 0, acc_v = 0, acc_p = 0;
  long long cnt = 0;
  R prev[VZ], cur[VZ], nxt[VZ], piC[VZ], piN[VZ];
#pragma unroll
  for (int k = 0; k < VZ; ++k) prev[k] = cur[k] = nxt[k] = piC[k] = piN[k] = R(0);
  if (x0 < x1) {
    // prologue: planes x0 - 1 .. x0 + L - 1 in flight; the first two into registers
#pragma unroll 1
    for (int j = 0; j <= L; ++j) issue(j);
    cp_async_wait<L - 1>();
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int k = 0; k < VZ; ++k) {
        prev[k] = fval(0, ctr + k);
        cur[k] = fval(1, ctr + k);
        if (LOADP) piC[k] = ringP[(1 % D) * PL + ctr + k];
      }
    }
#pragma unroll 1
    for (int x = x0; x < x1; ++x) {
      const int j = x - x0 + 1; // plane x's sequence index; x + 1 is j + 1
      cp_async_wait<L - 2>();   // planes up to x + 1 have landed (this thread's copies)
      __syncthreads();          // ... and every thread's; slot (j + L) % D = (j - 1) % D is free
      issue(j + L);
      if (valid) {
        const R *F = ringF + (j % D) * PL;
        const R *P = ringP + (j % D) * PL;
#pragma unroll
        for (int k = 0; k < VZ; ++k) {
          nxt[k] = fval(j + 1, ctr + k);
          if (LOADP) piN[k] = ringP[((j + 1) % D) * PL + ctr + k];
        }
        auto nb = [&](int e) -> R { return DRIFT ? drift_val<R>(F[e], P[e], pd, dtw) : F[e]; };
        const size_t s = sidx(x, y, z);
        R outp[VZ];
        if (DRIFT) stg_v<R, VZ>(fout + s, cur);
        if constexpr (SPLIT) {
          float s_p = 0.f, s_p2 = 0.f, s_g2 = 0.f, s_dv = 0.f;
#pragma unroll
          for (int k = 0; k < VZ; ++k) {
            const float c = cur[k];
            const float ynb = nb(ctr + ROW + k), ymb = nb(ctr - ROW + k);
            const float znb = k + 1 < VZ ? cur[k + 1 < VZ ? k + 1 : 0] : nb(ctr + VZ);
            const float zmb = k > 0 ? cur[k > 0 ? k - 1 : 0] : nb(ctr - 1);
            if (KICK) {
              const float lap = inv_dx2 * ((((nxt[k] + prev[k]) - 2.f * c) + ((ynb + ymb) - 2.f * c)) + ((znb + zmb) - 2.f * c));
              float ddv;
              if constexpr (kModelFluct) {
                ddv = spc.dV(c);
              } else {
                const double cd[1] = {rf.phi[0] + (double)c};
                ddv = (float)(SPot<double, 1>::dV(0, cd, lt.mc) - rf.dV[0]);
              }
              const float K = KA * lap - KB * ddv;
              const float pm = fmaf(h1f, K, piC[k]);
              outp[k] = h2f != 0.f ? fmaf(h2f, K, pm) : pm;
              if (RED & 1) {
                s_p += pm;
                s_p2 = fmaf(pm, pm, s_p2);
              }
            } else if (RED & 1) {
              s_p += piC[k];
              s_p2 = fmaf(piC[k], piC[k], s_p2);
            }
            if (RED & 2) {
              const float gx = nxt[k] - c, gy = ynb - c, gz = znb - c;
              s_g2 += (gx * gx + gy * gy + gz * gz) * inv_dx2;
              if constexpr (kModelFluct) {
                s_dv += spc.V(c);
              } else {
                const double cd[1] = {rf.phi[0] + (double)c};
                s_dv += (float)(SPot<double, 1>::V(cd, lt.mc) - rf.V);
              }
            }
          }
          acc_p += (double)s_p;
          acc_pi2 += (double)s_p2;
          acc_g2 += (double)s_g2;
          acc_v += (double)s_dv;
          cnt += VZ;
        } else {
#pragma unroll
          for (int k = 0; k < VZ; ++k) {
            const R c = cur[k];
            const R ynb = nb(ctr + ROW + k), ymb = nb(ctr - ROW + k);
            const R znb = k + 1 < VZ ? cur[k + 1 < VZ ? k + 1 : 0] : nb(ctr + VZ);
            const R zmb = k > 0 ? cur[k > 0 ? k - 1 : 0] : nb(ctr - 1);
            if (KICK) {
              const R txv = A::sub(A::add(nxt[k], prev[k]), A::mul(two, c));
              const R tyv = A::sub(A::add(ynb, ymb), A::mul(two, c));
              const R tzv = A::sub(A::add(znb, zmb), A::mul(two, c));
              const R lap = A::mul(inv_dx2, A::add(A::add(txv, tyv), tzv));
              const R cv[1] = {c};
              const R K = A::sub(A::mul(KA, lap), A::mul(KB, SPot<R, 1>::dV(0, cv, lt.mc)));
              const KickOut<R> ko = kick_val<R>(piC[k], K, h1, h2);
              outp[k] = ko.next;
              if (RED & 1) acc_pi2 += ko.mid * ko.mid;
            } else if (RED & 1) {
              acc_pi2 += (double)piC[k] * (double)piC[k];
            }
            if (RED & 2) {
              const R gx = A::sub(nxt[k], c), gy = A::sub(ynb, c), gz = A::sub(znb, c);
              acc_g2 += (double)A::mul(A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz)), inv_dx2);
              const R cv[1] = {c};
              acc_v += (double)SPot<R, 1>::V(cv, lt.mc);
            }
          }
        }
        if (KICK) stg_v<R, VZ>(pout + s, outp);
#pragma unroll
        for (int k = 0; k < VZ; ++k) {
          prev[k] = cur[k];
          cur[k] = nxt[k];
          piC[k] = piN[k];
        }
      }
    }
    cp_async_wait<0>(); // only empty groups remain past the run
  }
  if (RED) {
    if constexpr (SPLIT) {
      // sum (pi_r + p)^2 = n pi_r^2 + 2 pi_r sum p + sum p^2;  sum V = n V_r + sum (V - V_r)
      acc_pi2 += (double)cnt * rf.pi_mid[0] * rf.pi_mid[0] + 2.0 * rf.pi_mid[0] * acc_p;
      acc_v += (double)cnt * rf.V;
    }
    double v[kRedSlots] = {acc_pi2, acc_g2, acc_v};
    block_reduce<kRedSlots, BZ * BY>(v, red_smem);
#pragma unroll
    for (int k = 0; k < kRedSlots; ++k) vout[k] = v[k];
  }
  __syncthreads(); // the next tile of the same block reuses the ring and the scratch
}

template <int BZ, int BY, int VZ, class R, bool DRIFT, bool KICK, int RED>
__global__ void __launch_bounds__(BZ *BY, CLB_BATCH_MINB * 256 / (BZ * BY) / (VZ == 1 ? 1 : 2))
    k_batch_sweep(const R *fin, const R *pin, R *fout, R *pout, const BatchLat *__restrict__ lats,
                  const int *__restrict__ blk_lat, DevState *__restrict__ sts, int rs, double dtw_d, double h1,
                  double h2, double *__restrict__ partials)
{
  const int L = blk_lat[blockIdx.x];
  const BatchLat lt = lats[L];
  double v[kRedSlots] = {0, 0, 0};
  batch_tile<BZ, BY, VZ, R, DRIFT, KICK, RED>(fin, pin, fout, pout, lt, sts + L, blockIdx.x - lt.first_block, rs,
                                              dtw_d, h1, h2, v);
  if (RED && threadIdx.x == 0 && threadIdx.y == 0) {
#pragma unroll
    for (int k = 0; k < kRedSlots; ++k) partials[(size_t)blockIdx.x * kRedSlots + k] = v[k];
  }
}

// One block per member: fixed-order sum of the member's block partials, then the tail's
// scale-factor bookkeeping (tail_apply) on the member's DevState.
__global__ void __launch_bounds__(256)
    k_batch_tail(const double *__restrict__ partials, const BatchLat *__restrict__ lats, DevState *__restrict__ sts,
                 TailOp op, int reduced)
{
  __shared__ double smem[(256 / 32) * kRedSlots];
  const BatchLat lt = lats[blockIdx.x];
  double v[kRedSlots] = {0, 0, 0};
  if (reduced) {
    for (int b = threadIdx.x; b < lt.nblocks; b += blockDim.x) {
#pragma unroll
      for (int k = 0; k < kRedSlots; ++k) v[k] += partials[(size_t)(lt.first_block + b) * kRedSlots + k];
    }
    block_reduce<kRedSlots, 256>(v, smem);
  }
  if (threadIdx.x != 0) return;
  DevState s = sts[blockIdx.x];
  TailOp o = op;
  o.hist = nullptr;
  tail_apply(s, o, lt.sp, v[0], v[1], v[2]);
  sts[blockIdx.x] = s;
}

// ---- the whole evolve call as one persistent launch --------------------------------------------
// A thread-block cluster (CS CTAs, co-scheduled by the hardware) owns a list of members and takes
// each through every step of the call before the next: per stage its CTAs sweep their share of
// the member's tiles (tile t to CTA t % CS, in order), the cluster synchronises, CTA 0 adds the
// CTAs' sums in rank order through distributed shared memory and applies the member's
// scale-factor bookkeeping (tail_apply), and the cluster synchronises again before the next sweep
// reads the new state.  No CTA waits on another cluster: members are independent, and within a
// cluster every CTA runs the same loops and so the same barrier sequence.  The schedule is the
// graph form's (evolve_launches, clb_batch.cu): a first half kick, then one fused sweep per stage.
constexpr int kMaxStages = 31; // VV10

// One tile as its own (not inlined) function: the persistent kernel calls three tile variants, and
// inlined into its member and stage loops they would share one register allocation.
template <int BZ, int BY, int VZ, class R, bool DRIFT, bool KICK, int RED>
__device__ __noinline__ void persist_tile(const R *fin, const R *pin, R *fout, R *pout, const BatchLat &lt,
                                          DevState *st, int local, int rs, double dtw_d, double h1, double h2,
                                          double (&vout)[kRedSlots])
{
  batch_tile<BZ, BY, VZ, R, DRIFT, KICK, RED>(fin, pin, fout, pout, lt, st, local, rs, dtw_d, h1, h2, vout);
}

struct PersistArgs {
  double dt;
  int expansion;
  int stages;           // sweeps per step
  long long nsteps;
  double w[kMaxStages]; // stage weights
  int cf0, rs0;         // buffer parity and FP32 reference slot at the call's start (all members)
};

template <int BZ, int BY, int VZ, class R>
__global__ void __launch_bounds__(BZ *BY, CLB_BATCH_MINB * 256 / (BZ * BY) / (VZ == 1 ? 1 : 2))
    k_batch_persist(R *f0, R *p0, R *f1, R *p1, const BatchLat *__restrict__ lats, DevState *__restrict__ sts,
                    const int *__restrict__ members, const int *__restrict__ offsets, PersistArgs a)
{
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int crank = (int)cl.block_rank(), csize = (int)cl.num_blocks();
  const int cid = blockIdx.x / csize;
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  __shared__ double part[kRedSlots]; // this CTA's sums of the current stage
  R *F[2] = {f0, f1}, *P[2] = {p0, p1};
  const double dt = a.dt;
  for (int mi = offsets[cid]; mi < offsets[cid + 1]; ++mi) {
    const int L = members[mi];
    const BatchLat lt = lats[L];
    DevState *st = sts + L;
    int cf = a.cf0, rs = a.rs0;
    auto clear = [&]() {
      if (lead)
#pragma unroll
        for (int k = 0; k < kRedSlots; ++k) part[k] = 0.0;
    };
    auto add = [&](const double (&v)[kRedSlots]) {
      if (lead)
#pragma unroll
        for (int k = 0; k < kRedSlots; ++k) part[k] += v[k];
    };
    auto tail = [&](uint32_t flags, bool reduced, double w, double w2) {
      cl.sync(); // every CTA's sweep writes and sums are complete and visible
      if (crank == 0 && lead) {
        double v[kRedSlots] = {0, 0, 0};
        if (reduced)
          for (int r = 0; r < csize; ++r) {
            const double *pr = cl.map_shared_rank(part, r);
#pragma unroll
            for (int k = 0; k < kRedSlots; ++k) v[k] += pr[k];
          }
        DevState sv = *st;
        const TailOp op{flags, 0, w, w2, nullptr, -1, 0.0, 0.0};
        tail_apply(sv, op, lt.sp, v[0], v[1], v[2]);
        *st = sv;
      }
      cl.sync(); // the member's state is written before any CTA reads it, and `part` is free again
    };
    const int ntiles = lt.nblocks;
    const bool ex = a.expansion != 0;
    // the first half kick of the call (kickScaleFactorHalf, kickScalar, driftScaleFactor)
    if (ex) tail(T_VV_KICK_HALF, false, 0.0, a.w[0]);
    for (int t = crank; t < ntiles; t += csize) {
      double v[kRedSlots] = {0, 0, 0};
      persist_tile<BZ, BY, VZ, R, false, true, 0>(F[cf], P[cf], F[cf], P[cf], lt, st, t, rs, 0.0, a.w[0] * dt / 2, 0.0, v);
    }
    if (sizeof(R) == 4) rs ^= 1;
    if (ex)
      tail(T_VV_DRIFT, false, 0.0, a.w[0]);
    else
      cl.sync();
    const long long total = a.nsteps * a.stages;
    for (long long k = 0; k < total; ++k) {
      const int i = (int)(k % a.stages);
      const double w = a.w[i];
      const bool more = k + 1 < total;
      const double wn = more ? a.w[(int)((k + 1) % a.stages)] : 0.0;
      clear();
      for (int t = crank; t < ntiles; t += csize) {
        double v[kRedSlots] = {0, 0, 0};
        if (ex)
          persist_tile<BZ, BY, VZ, R, true, true, 3>(F[cf], P[cf], F[cf ^ 1], P[cf ^ 1], lt, st, t, rs, dt * w,
                                                   w * dt / 2, more ? wn * dt / 2 : 0.0, v);
        else
          persist_tile<BZ, BY, VZ, R, true, true, 0>(F[cf], P[cf], F[cf ^ 1], P[cf ^ 1], lt, st, t, rs, dt * w,
                                                   w * dt / 2, more ? wn * dt / 2 : 0.0, v);
        add(v);
      }
      cf ^= 1;
      if (sizeof(R) == 4) rs ^= 1;
      if (ex) {
        uint32_t fl = T_STORE_PI2_I | T_STORE_FIELDS | T_VV_KICK_ONE;
        if (more) fl |= T_VV_KICK_HALF | T_VV_DRIFT;
        tail(fl, true, w, wn);
      } else {
        cl.sync();
      }
    }
  }
}

// Host FP64 arrays <-> member storage: dst = (R)(src - off) and back (FP32: off = the member's
// reference value; FP64: off = 0).
template <class R>
__global__ void __launch_bounds__(256) k_batch_pack(const double *__restrict__ src, R *__restrict__ dst, size_t n, double off)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (R)(src[i] - off);
}
template <class R>
__global__ void __launch_bounds__(256) k_batch_unpack(const R *__restrict__ src, double *__restrict__ dst, size_t n, double off)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = off + (double)src[i];
}

// Measurement sums of one member (slots of k_measure: pi^2, grad^2, phi, phi^2, mom, mom^2, V),
// in FP64 from the stored values plus the member's references.
template <class R>
__global__ void __launch_bounds__(256)
    k_batch_measure(const R *__restrict__ f, const R *__restrict__ p, BatchLat lt, const DevState *__restrict__ st,
                    int rs, double am, double *__restrict__ partials)
{
  __shared__ double smem[(256 / 32) * 7];
  constexpr bool SPLIT = sizeof(R) == 4;
  const int N = lt.N;
  const size_t n3 = (size_t)N * N * N;
  f += lt.off;
  p += lt.off;
  const double fr = SPLIT ? st->ref_phi[rs][0] : 0.0, pr = SPLIT ? st->ref_pi[rs][0] : 0.0;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(s % N), y = (int)((s / N) % N), x = (int)(s / ((size_t)N * N));
    const size_t sx = ((size_t)(x + 1 == N ? 0 : x + 1) * N + y) * N + z;
    const size_t sy = ((size_t)x * N + (y + 1 == N ? 0 : y + 1)) * N + z;
    const size_t sz = ((size_t)x * N + y) * N + (z + 1 == N ? 0 : z + 1);
    const double c = fr + (double)f[s], pi = pr + (double)p[s];
    const double gx = (double)f[sx] - (double)f[s], gy = (double)f[sy] - (double)f[s], gz = (double)f[sz] - (double)f[s];
    const double m = pi * am;
    acc[0] += pi * pi;
    acc[1] += (gx * gx + gy * gy + gz * gz) * lt.inv_dx2;
    acc[2] += c;
    acc[3] += c * c;
    acc[4] += m;
    acc[5] += m * m;
    const double cv[1] = {c};
    acc[6] += SPot<double, 1>::V(cv, lt.mc);
  }
  block_reduce<7, 256>(acc, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < 7; ++k) partials[(size_t)blockIdx.x * 7 + k] = acc[k];
}

} // namespace clb
