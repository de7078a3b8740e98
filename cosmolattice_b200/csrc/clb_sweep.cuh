// clb_sweep.cuh - TMA-pipelined stencil sweeps over the padded (ghost-banded) lattice layout.
//
// Layout of one real component (Pad): N planes along x; each plane holds N+2 rows (one periodic
// ghost row on each side in y) of Zp elements (G ghost elements before z = 0, periodic ghosts at
// z = -1 and z = N, row pitch rounded up to 16 bytes).  Components are stacked plane after plane.
// With the ghosts in place every block's plane tile - its 64 x 8 (z, y) sites plus a halo of G
// columns and one row on each side - is an in-bounds box whose innermost start is 16-byte
// aligned, so one TMA instruction fetches it.  Each sweep also writes the z = -1, z = N, y = -1
// and y = N ghost copies of what it writes, so the next sweep's boxes are periodic again; elementwise
// updates keep ghosts consistent by updating them like interior sites.
//
// Sweep pipeline: thread 0 keeps up to S planes of phi (and pi) tiles in flight in a shared-memory
// ring (mbarrier completion with transaction counts); all 256 threads compute plane x from stages
// x and x+1 while planes x+2 ... x+S-1 stream in.  Each thread owns two adjacent z sites of one
// row; the x-1, x, x+1 centre values stay in registers.
#pragma once

#include "clb_internal.cuh"
#include "clb_scalar.cuh"
#include "clb_tma.cuh"

namespace clb {

struct Pad {
  int N, G, Zp, Yp;
  long long plane; // Yp * Zp elements
  long long comp;  // N * plane elements
  __host__ __device__ __forceinline__ long long at(int x, int y, int z) const
  {
    return (long long)x * plane + (long long)(y + 1) * Zp + (z + G);
  }
};

inline Pad make_pad(int N, int esz)
{
  Pad p;
  p.N = N;
  p.G = 16 / esz;
  const int q = 16 / esz;
  p.Zp = ((N + 2 * p.G + q - 1) / q) * q;
  p.Yp = N + 2;
  p.plane = (long long)p.Yp * p.Zp;
  p.comp = (long long)N * p.plane;
  return p;
}

// Block shape: TZ x TY threads, each owning VZ consecutive z sites of one row, so a block covers a
// (TZ VZ) x TY tile of (z, y) sites per plane.
template <int TZ_, int TY_, int VZ_> struct Shape {
  static constexpr int TZ = TZ_, TY = TY_, VZ = VZ_;
  static constexpr int BZ = TZ * VZ, BY = TY, THREADS = TZ * TY;
};
using ShapeW = Shape<32, 8, 2>;  // 64 x 8 sites, 2 per thread
using ShapeQ = Shape<16, 16, 4>; // 64 x 16 sites, 4 per thread
using ShapeH = Shape<16, 8, 4>;  // 64 x 8 sites, 4 per thread, 128 threads
using ShapeL = Shape<32, 8, 4>;  // 128 x 8 sites, 4 per thread, 256 threads
using ShapeK = Shape<32, 4, 4>;  // 128 x 4 sites, 4 per thread, 128 threads

template <class R, class SH> struct TileGeom {
  static constexpr int G = 16 / (int)sizeof(R);
  static constexpr int BOXZ = SH::BZ + 2 * G; // a 16-byte multiple
  static constexpr int BOXY = SH::BY + 2;
  static constexpr int BYTES = BOXZ * BOXY * (int)sizeof(R);
  static constexpr int SLOT = ((BYTES + 127) / 128) * 128; // TMA smem destinations 128-byte aligned
};

// Bound of each wait in a sweep's drain after an abort (copies already issued always complete).
constexpr uint32_t kDrainTries = 1u << 26;

template <bool B> struct BoolTag {
  static constexpr bool value = B;
};

struct SweepArgs {
  Pad pd;
  int LX;          // planes per block
  int S;           // ring stages
  int rs;          // FP32 split storage: reference slot read by this launch
  uint32_t tries;  // bound of each mbarrier wait
  double inv_dx2;
  CouplingSlot cs; // the model header's couplings (cs.mc)
  double dtw, h1, h2;
  double dtw0;     // DRIFT == 2: a first drift of the same kind before dtw's (position Verlet)
};

// VZ consecutive values from 16-byte-aligned shared memory.
template <class R, int VZ> __device__ __forceinline__ void ldv(const R *p, R (&v)[VZ])
{
  if constexpr (sizeof(R) == 8) {
#pragma unroll
    for (int k = 0; k < VZ; k += 2) {
      const double2 t = *reinterpret_cast<const double2 *>(p + k);
      v[k] = t.x;
      v[k + 1] = t.y;
    }
  } else if constexpr (VZ % 4 == 0) {
#pragma unroll
    for (int k = 0; k < VZ; k += 4) {
      const float4 t = *reinterpret_cast<const float4 *>(p + k);
      v[k] = t.x;
      v[k + 1] = t.y;
      v[k + 2] = t.z;
      v[k + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < VZ; k += 2) {
      const float2 t = *reinterpret_cast<const float2 *>(p + k);
      v[k] = t.x;
      v[k + 1] = t.y;
    }
  }
}

// VZ consecutive values to global memory at an address aligned to VZ elements (or 16 bytes).
template <class R, int VZ> __device__ __forceinline__ void stv(R *p, const R (&v)[VZ])
{
  if constexpr (sizeof(R) == 8) {
#pragma unroll
    for (int k = 0; k < VZ; k += 2) *reinterpret_cast<double2 *>(p + k) = double2{v[k], v[k + 1]};
  } else if constexpr (VZ % 4 == 0) {
#pragma unroll
    for (int k = 0; k < VZ; k += 4) *reinterpret_cast<float4 *>(p + k) = float4{v[k], v[k + 1], v[k + 2], v[k + 3]};
  } else {
#pragma unroll
    for (int k = 0; k < VZ; k += 2) *reinterpret_cast<float2 *>(p + k) = float2{v[k], v[k + 1]};
  }
}

// One VV sweep applied to the homogeneous FP64 references of the split storage: the same drift and
// kicks as a site with zero fluctuation (the Laplacian of a constant vanishes).
template <int NS> struct RefStep {
  double phi[NS], pi_mid[NS], pi_next[NS], dV[NS];
  double V; // potential at the reference point
};

// The model's FP32 fluctuation form (models/model_api.h), if its header has one: with one field,
// the force and energy of a fluctuation s about the FP64 reference, evaluated in FP32.  Without
// it (NoFluct) the split form takes both differences in FP64.
struct NoFluct {
  template <class C> __host__ __device__ static NoFluct make(double, const C &) { return {}; }
  __device__ float dV(float) const { return 0.f; } // never called: the FP64 differences are taken
  __device__ float V(float) const { return 0.f; }
};
template <class M, bool> struct FluctOf {
  using type = NoFluct;
};
template <class M> struct FluctOf<M, true> {
  using type = typename M::Fluct;
};
constexpr bool kModelFluct = clb_models::HasFluct<ScalarModel>::value;
using ModelFluct = typename FluctOf<ScalarModel, kModelFluct>::type;

template <int NS>
__device__ __forceinline__ RefStep<NS> ref_step(const DevState *st, int rs, bool drift, bool kick, double dtw, double h1,
                                                double h2, const ModelCouplings &mc, double dtw0 = 0.0)
{
  RefStep<NS> r;
  double phi[NS];
#pragma unroll
  for (int f = 0; f < NS; ++f) {
    phi[f] = st->ref_phi[rs][f];
    if (drift && dtw0 != 0.0) phi[f] = __dadd_rn(phi[f], __dmul_rn(st->drift_p, __dmul_rn(dtw0, st->ref_pi[rs][f])));
    if (drift) phi[f] = __dadd_rn(phi[f], __dmul_rn(st->drift_p, __dmul_rn(dtw, st->ref_pi[rs][f])));
    r.phi[f] = phi[f];
  }
  r.V = SPot<double, NS>::V(phi, mc);
#pragma unroll
  for (int f = 0; f < NS; ++f) {
    r.dV[f] = SPot<double, NS>::dV(f, phi, mc);
    const double Kr = -__dmul_rn(st->kick_B, r.dV[f]);
    const double p0 = st->ref_pi[rs][f];
    r.pi_mid[f] = kick ? __dadd_rn(p0, __dmul_rn(h1, Kr)) : p0;
    r.pi_next[f] = (kick && h2 != 0.0) ? __dadd_rn(r.pi_mid[f], __dmul_rn(h2, Kr)) : r.pi_mid[f];
  }
  return r;
}

// DRIFT / KICK / RED as in k_scalar_sweep (clb_scalar.cuh), with DRIFT == 2 two successive drifts
// (dtw0, then dtw) each rounded as the reference's (the end drift of a position-Verlet stage and the
// first drift of the next); fout/pout are padded arrays.
// FP32 storage holds fluctuations around the FP64 references (DevState::ref_*): FP32 arithmetic on
// the fluctuations, with the reference terms of the volume sums added in FP64.
template <class R, int NS, class SH, int DRIFT, bool KICK, int RED>
__global__ void __launch_bounds__(SH::THREADS)
    k_sweep(const __grid_constant__ CUtensorMap tmf, const __grid_constant__ CUtensorMap tmp, R *fout, R *pout,
            SweepArgs a, const DevState *__restrict__ st, double *__restrict__ partials, int *__restrict__ err)
{
  using A = Ar<R>;
  using Pot = SPot<R, NS>;
  using TG = TileGeom<R, SH>;
  constexpr int VZ = SH::VZ;
  constexpr bool LOADP = DRIFT || KICK || (RED & 1);
  constexpr int NB = LOADP ? 2 : 1;
  constexpr int BOXZ = TG::BOXZ;
  constexpr bool SPLIT = sizeof(R) == 4;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int S = a.S;
  const size_t stage_bytes = (size_t)NS * NB * TG::SLOT;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)S * stage_bytes);
  double *red_smem = reinterpret_cast<double *>(bars + S);
  __shared__ int abort_flag;

  const Pad &pd = a.pd;
  const int N = pd.N;
  const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * SH::TZ + tz;
  const int z0 = blockIdx.x * SH::BZ, y0 = blockIdx.y * SH::BY;
  const int x0 = blockIdx.z * a.LX, x1 = min(N, x0 + a.LX);
  const int z = z0 + VZ * tz, y = y0 + ty;
  const bool vy = y < N;
  const int nvalid = vy ? max(0, min(VZ, N - z)) : 0; // sites of this thread inside the lattice
  const int toff = (ty + 1) * BOXZ + TG::G + VZ * tz; // box offset of site 0
  const int nplanes = x1 - x0 + 2;                     // planes x0-1 .. x1
  const uint32_t tx_bytes = (uint32_t)(NS * NB * TG::BYTES);

  // Independent of the preceding kernels: barrier set-up and tensor-map prefetch.  Everything after
  // griddep_wait may read what they wrote (state arrays, DevState) or overwrite what they read
  // (partials, the DevState reference slot).
  if (tid == 0) {
    abort_flag = 0;
    prefetch_tensormap(&tmf);
    if (LOADP) prefetch_tensormap(&tmp);
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  griddep_wait();

  if (x0 >= x1) { // block-uniform: no planes, but its partial row must not hold stale sums
    if (RED && tid == 0) {
      const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
      for (int k = 0; k < kRedSlots; ++k) partials[bid * kRedSlots + k] = 0.0;
    }
    return;
  }

  R pdr = R(0), dtw = R(0), dtw0 = R(0), KA = R(0), KB = R(0);
  if (DRIFT) {
    pdr = (R)st->drift_p;
    dtw = (R)a.dtw;
    if (DRIFT == 2) dtw0 = (R)a.dtw0;
  }
  if (KICK) {
    KA = (R)st->kick_A;
    KB = (R)st->kick_B;
  }
  const R inv_dx2 = (R)a.inv_dx2;
  const R two = R(2);
  RefStep<NS> rf{};
  ModelFluct spc{};
  const float h1f = (float)a.h1, h2f = (float)a.h2;
  if constexpr (SPLIT) {
    rf = ref_step<NS>(st, a.rs, DRIFT, KICK, a.dtw, a.h1, a.h2, a.cs.mc, DRIFT == 2 ? a.dtw0 : 0.0);
    spc = ModelFluct::make(rf.phi[0], a.cs.mc);
    if ((DRIFT || KICK) && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && tid == 0) {
      DevState *sw = const_cast<DevState *>(st); // slot rs ^ 1 is read by no block of this launch
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        sw->ref_phi[a.rs ^ 1][f] = rf.phi[f];
        sw->ref_pi[a.rs ^ 1][f] = rf.pi_next[f];
      }
    }
  }

  // box (stage s, field f, k = 0 phi / 1 pi)
  auto box = [&](int s, int f, int k) -> R * {
    return reinterpret_cast<R *>(smem_raw + (size_t)s * stage_bytes + (size_t)(f * NB + k) * TG::SLOT);
  };
  auto issue = [&](int j) { // plane ring index j -> lattice plane x0 - 1 + j (periodic)
    const int s = j % S;
    int p = x0 - 1 + j;
    p = p < 0 ? p + N : (p >= N ? p - N : p);
    mbar_arrive_expect_tx(&bars[s], tx_bytes);
#pragma unroll
    for (int f = 0; f < NS; ++f) {
      tma_load_3d(box(s, f, 0), &tmf, &bars[s], z0, y0, f * N + p);
      if (LOADP) tma_load_3d(box(s, f, 1), &tmp, &bars[s], z0, y0, f * N + p);
    }
  };
  auto drift1 = [&](R phi, R pi) -> R {
    if (DRIFT == 2) return drift_val<R>(drift_val<R>(phi, pi, pdr, dtw0), pi, pdr, dtw);
    return DRIFT ? drift_val<R>(phi, pi, pdr, dtw) : phi;
  };
  // VZ drifted values at box offset o of stage s, field f (and the raw pi values if wanted)
  auto dquad = [&](int s, int f, int o, R (&out)[VZ], R (*praw)[VZ]) {
    R fv[VZ];
    ldv<R, VZ>(box(s, f, 0) + o, fv);
    if (LOADP) {
      R pv[VZ];
      ldv<R, VZ>(box(s, f, 1) + o, pv);
#pragma unroll
      for (int k = 0; k < VZ; ++k) out[k] = drift1(fv[k], pv[k]);
      if (praw)
#pragma unroll
        for (int k = 0; k < VZ; ++k) (*praw)[k] = pv[k];
    } else {
#pragma unroll
      for (int k = 0; k < VZ; ++k) out[k] = fv[k];
    }
  };
  auto dscalar = [&](int s, int f, int o) -> R {
    const R fv = box(s, f, 0)[o];
    return LOADP ? drift1(fv, box(s, f, 1)[o]) : fv;
  };
  // neighbour values of the current plane (stage s): y - 1, y + 1 rows and the z - 1, z + VZ cells,
  // each drifted as it is read (a drift of each plane once, written back to shared memory by its
  // owners, measured no faster: the stores and the halo work cost what the drifts saved)
  auto neighbours = [&](int s, int f, R (&ym)[VZ], R (&yp)[VZ], R &zm, R &zp) {
    dquad(s, f, toff - BOXZ, ym, nullptr);
    dquad(s, f, toff + BOXZ, yp, nullptr);
    zm = dscalar(s, f, toff - 1);
    zp = dscalar(s, f, toff + VZ);
  };

  __syncthreads();
  if (tid == 0)
    for (int j = 0; j < min(S, nplanes); ++j) issue(j);

  // Thread 0 tracks the planes issued and the first plane whose wait did not complete, for the
  // drain on abort: a wait that gave up leaves its copy in flight.
  // Plane j sits in ring stage j % S with barrier parity (j / S) & 1; the loop keeps both as running
  // counters (no division by the run-time ring depth per plane).
  int issued = min(S, nplanes), waited = 0;
  bool gave_up = false;
  auto wait_plane = [&](int j, int stage, uint32_t parity) {
    if (!mbar_wait(&bars[stage], parity, a.tries)) {
      abort_flag = 1;
      gave_up = true;
    }
    if (tid == 0 && !gave_up) waited = j + 1;
  };

  // periodic ghost copies this thread writes (they depend on y and z only): y row -1 / N, z column -1 / N
  const long long ioff = (long long)(y + 1) * pd.Zp + (z + pd.G); // offset of site 0 inside a plane
  const int ghost_y = (y == 0) ? N : (y == N - 1 ? -1 : -2);     // target row, -2: none
  const int kz_first = z == 0 ? 0 : -1;                         // site writing the z = N ghost
  const int kz_last = (N - 1 - z >= 0 && N - 1 - z < nvalid) ? N - 1 - z : -1; // site writing z = -1
  const bool has_ghost = nvalid > 0 && (ghost_y != -2 || kz_first >= 0 || kz_last >= 0);

  R prev[NS][VZ], cur[NS][VZ], nxt[NS][VZ], piC[NS][VZ], piN[NS][VZ];
  wait_plane(0, 0, 0u); // S >= 3: planes 0, 1 and 2 are in stages 0, 1 and 2 of the first lap
#pragma unroll
  for (int f = 0; f < NS; ++f) dquad(0, f, toff, prev[f], nullptr);
  wait_plane(1, 1, 0u);
#pragma unroll
  for (int f = 0; f < NS; ++f) {
    dquad(1, f, toff, cur[f], LOADP ? &piC[f] : nullptr);
  }
  __syncthreads();
  if (abort_flag) goto drain;
  if (tid == 0 && S < nplanes) {
    issue(S);
    issued = S + 1;
  }

  {
    double acc_pi2 = 0, acc_g2 = 0, acc_v = 0;
    double acc_p[NS]; // FP32 split: sum of the momentum fluctuation per field
#pragma unroll
    for (int f = 0; f < NS; ++f) acc_p[f] = 0;
    long long cnt = 0; // FP32 split: sites summed by this thread
    long long pbase = (long long)x0 * pd.plane;
    int sb = 1, sn = 2;  // stages of planes j and j + 1
    uint32_t par_n = 0u; // barrier parity of plane j + 1
    for (int x = x0; x < x1; ++x, pbase += pd.plane) {
      const int j = x - x0 + 1;
      // the drifted plane x is known here: store it first, so the registers are free long before
      // the rotation below overwrites them
      if (DRIFT && nvalid == VZ)
#pragma unroll
        for (int f = 0; f < NS; ++f) stv<R, VZ>(fout + ((long long)f * pd.comp + pbase + ioff), cur[f]);
      wait_plane(j + 1, sn, par_n);
      R ym[NS][VZ], yp[NS][VZ], zmv[NS], zpv[NS];
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        dquad(sn, f, toff, nxt[f], LOADP ? &piN[f] : nullptr);
        neighbours(sb, f, ym[f], yp[f], zmv[f], zpv[f]);
      }
      R outp[NS][VZ];
      if constexpr (SPLIT) {
        // Full tiles (every site of the thread inside the lattice) take a copy of the plane's
        // arithmetic without the per-site predicates of the volume sums.
        auto split_plane = [&](auto full_tag) {
          constexpr bool FULL = decltype(full_tag)::value;
          // FP32 fluctuations about the FP64 references: FP32 arithmetic throughout, per-plane FP32
          // partial sums folded into FP64 accumulators (the reference terms are added at the end).
          // Not bound to the reference's operation order: the Laplacian is (sum of the six
          // neighbours) - 6 c with 1/dx^2 folded into the kick coefficient, and the gradient sum is
          // scaled once per plane.
          float s_p[NS], s_p2 = 0.f, s_g2 = 0.f, s_dv = 0.f;
          const float KAd = KA * inv_dx2;
#pragma unroll
          for (int f = 0; f < NS; ++f) s_p[f] = 0.f;
#pragma unroll
          for (int k = 0; k < VZ; ++k) {
            const bool vk = FULL || k < nvalid; // FULL: every site of the thread is inside
            float cv[NS];
            constexpr bool FL = NS == 1 && kModelFluct; // the header's FP32 fluctuation form
            double cd[NS];                                // otherwise the full field values in FP64
#pragma unroll
            for (int f = 0; f < NS; ++f) {
              cv[f] = cur[f][k];
              if constexpr (!FL) cd[f] = rf.phi[f] + (double)cur[f][k];
            }
            (void)cd;
#pragma unroll
            for (int f = 0; f < NS; ++f) {
              const float c = cur[f][k];
              const float zn = k + 1 < VZ ? cur[f][k + 1 < VZ ? k + 1 : 0] : zpv[f];
              const float zm = k > 0 ? cur[f][k > 0 ? k - 1 : 0] : zmv[f];
              if (KICK) {
                const float nsum = ((nxt[f][k] + prev[f][k]) + (yp[f][k] + ym[f][k])) + (zn + zm);
                const float lap = fmaf(-6.f, c, nsum); // times 1/dx^2 in KAd
                float ddv;
                if constexpr (FL)
                  ddv = spc.dV(c);
                else
                  ddv = (float)(SPot<double, NS>::dV(f, cd, a.cs.mc) - rf.dV[f]);
                const float K = KAd * lap - KB * ddv;
                const float pm = fmaf(h1f, K, piC[f][k]);
                outp[f][k] = h2f != 0.f ? fmaf(h2f, K, pm) : pm;
                if ((RED & 1) && vk) {
                  s_p[f] += pm;
                  s_p2 = fmaf(pm, pm, s_p2);
                }
              } else if ((RED & 1) && vk) {
                s_p[f] += piC[f][k];
                s_p2 = fmaf(piC[f][k], piC[f][k], s_p2);
              }
              if ((RED & 2) && vk) {
                const float gx = nxt[f][k] - c, gy = yp[f][k] - c, gz = zn - c;
                s_g2 += gx * gx + gy * gy + gz * gz; // times 1/dx^2 per plane
              }
            }
            if ((RED & 2) && vk) {
              if constexpr (FL)
                s_dv += spc.V(cv[0]);
              else
                s_dv += (float)(SPot<double, NS>::V(cd, a.cs.mc) - rf.V);
            }
          }
          if (RED) {
#pragma unroll
            for (int f = 0; f < NS; ++f) acc_p[f] += (double)s_p[f];
            acc_pi2 += (double)s_p2;
            acc_g2 += (double)s_g2 * a.inv_dx2;
            acc_v += (double)s_dv;
            cnt += nvalid;
          }
        };
        if (nvalid == VZ)
          split_plane(BoolTag<true>{});
        else
          split_plane(BoolTag<false>{});
      } else {
#pragma unroll
      for (int k = 0; k < VZ; ++k) {
        R cv[NS];
#pragma unroll
        for (int f = 0; f < NS; ++f) cv[f] = cur[f][k];
        double site_pi2 = 0;
#pragma unroll
        for (int f = 0; f < NS; ++f) {
          const R c = cur[f][k];
          const R zn = k + 1 < VZ ? cur[f][k + 1 < VZ ? k + 1 : 0] : zpv[f];
          const R zm = k > 0 ? cur[f][k > 0 ? k - 1 : 0] : zmv[f];
          if (KICK) {
            const R txv = A::sub(A::add(nxt[f][k], prev[f][k]), A::mul(two, c));
            const R tyv = A::sub(A::add(yp[f][k], ym[f][k]), A::mul(two, c));
            const R tzv = A::sub(A::add(zn, zm), A::mul(two, c));
            const R lap = A::mul(inv_dx2, A::add(A::add(txv, tyv), tzv));
            const R K = A::sub(A::mul(KA, lap), A::mul(KB, Pot::dV(f, cv, a.cs.mc)));
            const KickOut<R> ko = kick_val<R>(piC[f][k], K, a.h1, a.h2);
            outp[f][k] = ko.next;
            if (RED & 1) site_pi2 = f == 0 ? ko.mid * ko.mid : site_pi2 + ko.mid * ko.mid;
          } else if (RED & 1) {
            const double pc = (double)piC[f][k];
            site_pi2 = f == 0 ? pc * pc : site_pi2 + pc * pc;
          }
          if ((RED & 2) && k < nvalid) {
            const R gx = A::sub(nxt[f][k], c), gy = A::sub(yp[f][k], c), gz = A::sub(zn, c);
            acc_g2 += (double)A::mul(A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz)), inv_dx2);
          }
        }
        if ((RED & 1) && k < nvalid) acc_pi2 += site_pi2;
        if ((RED & 2) && k < nvalid) acc_v += (double)Pot::V(cv, a.cs.mc);
      }
      }
      // stores: the thread's VZ sites, then the periodic ghost copies of boundary sites
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        const long long o = (long long)f * pd.comp + pbase + ioff;
        if (nvalid == VZ) {
          if (KICK) stv<R, VZ>(pout + o, outp[f]); // fields stored at the top of the iteration
        } else {
#pragma unroll
          for (int k = 0; k < VZ; ++k)
            if (k < nvalid) {
              if (DRIFT) fout[o + k] = cur[f][k];
              if (KICK) pout[o + k] = outp[f][k];
            }
        }
        if (has_ghost) {
          const long long fp = (long long)f * pd.comp + pbase;
#pragma unroll
          for (int k = 0; k < VZ; ++k) {
            if (k >= nvalid) continue;
            long long g[3];
            int ng = 0;
            if (ghost_y != -2) g[ng++] = fp + pd.at(0, ghost_y, z + k);
            if (k == kz_first) g[ng++] = fp + pd.at(0, y, N);
            if (k == kz_last) g[ng++] = fp + pd.at(0, y, -1);
            for (int i = 0; i < ng; ++i) {
              if (DRIFT) fout[g[i]] = cur[f][k];
              if (KICK) pout[g[i]] = outp[f][k];
            }
          }
        }
      }
      __syncthreads(); // stage sb fully read
      if (abort_flag) goto drain;
      if (tid == 0 && j + S < nplanes) {
        issue(j + S);
        issued = j + S + 1;
      }
#pragma unroll
      for (int f = 0; f < NS; ++f)
#pragma unroll
        for (int k = 0; k < VZ; ++k) {
          prev[f][k] = cur[f][k];
          cur[f][k] = nxt[f][k];
          if (LOADP) piC[f][k] = piN[f][k];
        }
      sb = sn;
      if (++sn == S) {
        sn = 0;
        par_n ^= 1u;
      }
    }
    griddep_launch(); // planes done: the tail may be scheduled
    if (RED) {
      if constexpr (SPLIT) {
        // sum (pi_r + p)^2 = n pi_r^2 + 2 pi_r sum p + sum p^2;  sum V = n V_r + sum (V - V_r)
        double t = acc_pi2;
#pragma unroll
        for (int f = 0; f < NS; ++f) t += (double)cnt * rf.pi_mid[f] * rf.pi_mid[f] + 2.0 * rf.pi_mid[f] * acc_p[f];
        acc_pi2 = t;
        acc_v += (double)cnt * rf.V;
      }
      double v[kRedSlots] = {acc_pi2, acc_g2, acc_v};
      block_reduce<kRedSlots, SH::THREADS>(v, red_smem);
      if (tid == 0) {
        const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
        for (int k = 0; k < kRedSlots; ++k) partials[bid * kRedSlots + k] = v[k];
      }
    }
    return;
  }

drain:
  // A wait gave up: flag it, then let thread 0 wait for the copies still in flight so no TMA write
  // lands in shared memory after the block has left.  The drain has its own fixed bound, far above
  // the time a tile load takes, so a small a.tries cannot cut it short.
  if (tid == 0) {
    atomicOr(err, 1);
    for (int j = waited; j < issued; ++j) (void)mbar_wait(&bars[j % S], (uint32_t)((j / S) & 1), kDrainTries);
  }
}

// ---- padded elementwise / row kernels -------------------------------------------------------------
// Sum over interior sites of sum_f pi_f^2 into slot 0 of each block's partial row.
template <class R, int NS>
__global__ void __launch_bounds__(256)
    k_reduce_pi2_pad(const R *pi, Pad pd, const DevState *__restrict__ st, int rs, double *__restrict__ partials)
{
  __shared__ double smem[(256 / 32) * kRedSlots];
  const int N = pd.N;
  double pref[NS];
#pragma unroll
  for (int f = 0; f < NS; ++f) pref[f] = sizeof(R) == 4 ? st->ref_pi[rs][f] : 0.0;
  double acc = 0;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int x = (int)(r / N), y = (int)(r % N);
    for (int z = threadIdx.x; z < N; z += blockDim.x) {
      const long long s = pd.at(x, y, z);
      double v = 0;
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        const double p = sizeof(R) == 4 ? pref[f] + (double)pi[f * pd.comp + s] : (double)pi[f * pd.comp + s];
        v = f == 0 ? p * p : v + p * p;
      }
      acc += v;
    }
  }
  double v[kRedSlots] = {acc, 0.0, 0.0};
  block_reduce<kRedSlots, 256>(v, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < kRedSlots; ++k) partials[(size_t)blockIdx.x * kRedSlots + k] = v[k];
}

// Measurement sums (same slots as k_measure) over the padded layout.
template <class R, int NS>
__global__ void __launch_bounds__(256)
    k_measure_pad(const R *fld, const R *pi, Pad pd, double inv_dx2d, ModelCouplings mc, double am,
                  const DevState *__restrict__ st, int rs, double *__restrict__ partials)
{
  constexpr bool SPLIT = sizeof(R) == 4;
  using A = Ar<R>;
  using Pot = SPot<R, NS>;
  __shared__ double smem[(256 / 32) * kMeasSlots];
  const int N = pd.N;
  const R inv_dx2 = (R)inv_dx2d;
  double acc[kMeasSlots];
#pragma unroll
  for (int k = 0; k < kMeasSlots; ++k) acc[k] = 0;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int x = (int)(r / N), y = (int)(r % N);
    const int xp = x + 1 == N ? 0 : x + 1;
    for (int z = threadIdx.x; z < N; z += blockDim.x) {
      const long long s = pd.at(x, y, z);
      const long long sx = pd.at(xp, y, z), sy = pd.at(x, y + 1, z), sz = pd.at(x, y, z + 1);
      R v[NS];
      double vd[NS];
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        const long long o = f * pd.comp;
        const R c = fld[o + s];
        v[f] = c;
        const double cfull = SPLIT ? st->ref_phi[rs][f] + (double)c : (double)c;
        vd[f] = cfull;
        const R gx = A::sub(fld[o + sx], c), gy = A::sub(fld[o + sy], c), gz = A::sub(fld[o + sz], c);
        const R g2 = A::mul(A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz)), inv_dx2);
        const double p = SPLIT ? st->ref_pi[rs][f] + (double)pi[o + s] : (double)pi[o + s];
        const double m = p * am;
        acc[6 * f + 0] += p * p;
        acc[6 * f + 1] += (double)g2;
        acc[6 * f + 2] += cfull;
        acc[6 * f + 3] += cfull * cfull;
        acc[6 * f + 4] += m;
        acc[6 * f + 5] += m * m;
      }
#pragma unroll
      for (int k = 0; k < NS; ++k)
        acc[6 * NS + k] += SPLIT ? SPot<double, NS>::Vterm(k, vd, mc) : (double)Pot::Vterm(k, v, mc);
    }
  }
  block_reduce<kMeasSlots, 256>(acc, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < kMeasSlots; ++k) partials[(size_t)blockIdx.x * kMeasSlots + k] = acc[k];
}

// Host-order planes (plane p = f N + x, N x N each) -> padded interior, with type conversion.
// Per-component constant removed on upload and added back on download (FP32 split references).
struct CompOffsets {
  double v[2];
};

template <class S, class D>
__global__ void __launch_bounds__(256)
    k_scatter(const S *__restrict__ src, D *__restrict__ dst, Pad pd, long long p0, long long np, CompOffsets off)
{
  const int N = pd.N;
  for (long long r = blockIdx.x; r < np * N; r += gridDim.x) {
    const long long p = p0 + r / N;
    const int y = (int)(r % N);
    const int f = (int)(p / N), x = (int)(p % N);
    const long long o = (long long)f * pd.comp + pd.at(x, y, 0);
    const double c = off.v[f];
    for (int z = threadIdx.x; z < N; z += blockDim.x) dst[o + z] = (D)((double)src[r * N + z] - c);
  }
}

template <class S, class D>
__global__ void __launch_bounds__(256)
    k_gather(const S *__restrict__ src, D *__restrict__ dst, Pad pd, long long p0, long long np, CompOffsets off)
{
  const int N = pd.N;
  for (long long r = blockIdx.x; r < np * N; r += gridDim.x) {
    const long long p = p0 + r / N;
    const int y = (int)(r % N);
    const int f = (int)(p / N), x = (int)(p % N);
    const long long o = (long long)f * pd.comp + pd.at(x, y, 0);
    const double c = off.v[f];
    for (int z = threadIdx.x; z < N; z += blockDim.x) dst[r * N + z] = (D)(c + (double)src[o + z]);
  }
}

// Periodic ghost copies: rows y = -1, N and columns z = -1, N of every plane of every component.
template <class R> __global__ void __launch_bounds__(256) k_fill_ghosts(R *a, Pad pd, int ncomp)
{
  const int N = pd.N;
  const long long per_plane = 4LL * N;
  const long long total = (long long)ncomp * N * per_plane;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long pl = i / per_plane;
    const int t = (int)(i % per_plane);
    const int f = (int)(pl / N), x = (int)(pl % N);
    R *c = a + (long long)f * pd.comp;
    if (t < 2 * N) {
      const int zz = t % N;
      if (t < N) c[pd.at(x, -1, zz)] = c[pd.at(x, N - 1, zz)];
      else c[pd.at(x, N, zz)] = c[pd.at(x, 0, zz)];
    } else {
      const int u = t - 2 * N, yy = u % N;
      if (u < N) c[pd.at(x, yy, -1)] = c[pd.at(x, yy, N - 1)];
      else c[pd.at(x, yy, N)] = c[pd.at(x, yy, 0)];
    }
  }
}

} // namespace clb
