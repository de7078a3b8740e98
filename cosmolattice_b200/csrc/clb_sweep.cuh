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

constexpr int kTZ = 32, kTY = 8, kVZ = 2;
constexpr int kTileZ = kTZ * kVZ; // 64 z sites per block
constexpr int kSweepThreads = kTZ * kTY;

template <class R> struct TileGeom {
  static constexpr int G = 16 / (int)sizeof(R);
  static constexpr int BOXZ = kTileZ + 2 * G; // 68 (FP64) / 72 (FP32): 16-byte multiple
  static constexpr int BOXY = kTY + 2;
  static constexpr int BYTES = BOXZ * BOXY * (int)sizeof(R);
  static constexpr int SLOT = ((BYTES + 127) / 128) * 128; // TMA smem destinations 128-byte aligned
};

struct SweepArgs {
  Pad pd;
  int LX;          // planes per block
  int S;           // ring stages
  uint32_t tries;  // bound of each mbarrier wait
  double inv_dx2, c0, q, c0_quarter, q_half;
  double dtw, h1, h2;
};

template <class R> struct Vec2;
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<float> { using T = float2; };

template <class R, int NS> constexpr int sweep_boxes(bool loadp) { return NS * (loadp ? 2 : 1); }

// DRIFT / KICK / RED as in k_scalar_sweep (clb_scalar.cuh); fout/pout are padded arrays.
template <class R, int NS, bool DRIFT, bool KICK, int RED>
__global__ void __launch_bounds__(kSweepThreads)
    k_sweep(const __grid_constant__ CUtensorMap tmf, const __grid_constant__ CUtensorMap tmp, R *fout, R *pout,
            SweepArgs a, const DevState *__restrict__ st, double *__restrict__ partials, int *__restrict__ err)
{
  using A = Ar<R>;
  using Pot = Lphi4<R, NS>;
  using TG = TileGeom<R>;
  using V2 = typename Vec2<R>::T;
  constexpr bool LOADP = DRIFT || KICK || (RED & 1);
  constexpr int NB = LOADP ? 2 : 1;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int S = a.S;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)S * NS * NB * TG::SLOT);
  double *red_smem = reinterpret_cast<double *>(bars + S);
  __shared__ int abort_flag;

  const Pad &pd = a.pd;
  const int N = pd.N;
  const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * kTZ + tz;
  const int z0 = blockIdx.x * kTileZ, y0 = blockIdx.y * kTY;
  const int x0 = blockIdx.z * a.LX, x1 = min(N, x0 + a.LX);
  const int zl = kVZ * tz;
  const int z = z0 + zl, y = y0 + ty;
  const bool vy = y < N;
  const bool v0 = vy && z < N, v1 = vy && z + 1 < N;
  const int row = ty + 1, col = TG::G + zl;
  const int nplanes = x1 - x0 + 2; // planes x0-1 .. x1
  const uint32_t tx_bytes = (uint32_t)(NS * NB * TG::BYTES);

  R pdr = R(0), dtw = R(0), KA = R(0), KB = R(0);
  if (DRIFT) {
    pdr = (R)st->drift_p;
    dtw = (R)a.dtw;
  }
  if (KICK) {
    KA = (R)st->kick_A;
    KB = (R)st->kick_B;
  }
  const R inv_dx2 = (R)a.inv_dx2;
  const R c0 = (R)a.c0, q = (R)a.q, c0q = (R)a.c0_quarter, qh = (R)a.q_half;
  const R two = R(2);

  auto box = [&](int s, int f, int k) -> R * {
    return reinterpret_cast<R *>(smem_raw + ((size_t)(s * NS + f) * NB + k) * TG::SLOT);
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
  auto dval = [&](int s, int f, int r, int c) -> R {
    R v = box(s, f, 0)[r * TG::BOXZ + c];
    if (DRIFT) v = drift_val<R>(v, box(s, f, 1)[r * TG::BOXZ + c], pdr, dtw);
    return v;
  };

  if (x0 >= x1) { // block-uniform: no planes, but its partial row must not hold stale sums
    if (RED && tid == 0) {
      const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
      for (int k = 0; k < kRedSlots; ++k) partials[bid * kRedSlots + k] = 0.0;
    }
    return;
  }
  if (tid == 0) {
    abort_flag = 0;
    prefetch_tensormap(&tmf);
    if (LOADP) prefetch_tensormap(&tmp);
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0)
    for (int j = 0; j < min(S, nplanes); ++j) issue(j);

  int issued = min(S, nplanes), waited = 0; // tracked by thread 0 for the drain on abort
  auto wait_plane = [&](int j) {
    if (!mbar_wait(&bars[j % S], (uint32_t)((j / S) & 1), a.tries)) abort_flag = 1;
    if (tid == 0) waited = j + 1;
  };

  R prev[NS][2], cur[NS][2], nxt[NS][2], piC[NS][2], piN[NS][2];
  wait_plane(0);
#pragma unroll
  for (int f = 0; f < NS; ++f)
#pragma unroll
    for (int k = 0; k < 2; ++k) prev[f][k] = dval(0, f, row, col + k);
  wait_plane(1);
#pragma unroll
  for (int f = 0; f < NS; ++f)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      cur[f][k] = dval(1 % S, f, row, col + k);
      if (LOADP) piC[f][k] = box(1 % S, f, 1)[row * TG::BOXZ + col + k];
    }
  __syncthreads();
  if (abort_flag) goto drain;
  if (tid == 0 && S < nplanes) {
    issue(S);
    issued = S + 1;
  }

  {
    double acc_pi2 = 0, acc_g2 = 0, acc_v = 0;
    for (int x = x0; x < x1; ++x) {
      const int j = x - x0 + 1;
      const int sb = j % S, sn = (j + 1) % S;
      wait_plane(j + 1);
#pragma unroll
      for (int f = 0; f < NS; ++f)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          nxt[f][k] = dval(sn, f, row, col + k);
          if (LOADP) piN[f][k] = box(sn, f, 1)[row * TG::BOXZ + col + k];
        }
      // in-plane neighbours of plane x (drifted), per field: y-1 and y+1 pairs, z-1 of site 0, z+1 of site 1
      R ym[NS][2], yp[NS][2], zm0[NS], zp1[NS];
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        ym[f][0] = dval(sb, f, row - 1, col);
        ym[f][1] = dval(sb, f, row - 1, col + 1);
        yp[f][0] = dval(sb, f, row + 1, col);
        yp[f][1] = dval(sb, f, row + 1, col + 1);
        zm0[f] = dval(sb, f, row, col - 1);
        zp1[f] = dval(sb, f, row, col + 2);
      }
      const long long base = pd.at(x, y, z);
      R outf[NS][2], outp[NS][2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const bool vk = k == 0 ? v0 : v1;
        R cv[NS];
#pragma unroll
        for (int f = 0; f < NS; ++f) cv[f] = cur[f][k];
        double site_pi2 = 0;
#pragma unroll
        for (int f = 0; f < NS; ++f) {
          const R c = cur[f][k];
          const R zn = k == 0 ? cur[f][1] : zp1[f];
          const R zmv = k == 0 ? zm0[f] : cur[f][0];
          outf[f][k] = c;
          if (KICK) {
            const R txv = A::sub(A::add(nxt[f][k], prev[f][k]), A::mul(two, c));
            const R tyv = A::sub(A::add(yp[f][k], ym[f][k]), A::mul(two, c));
            const R tzv = A::sub(A::add(zn, zmv), A::mul(two, c));
            const R lap = A::mul(inv_dx2, A::add(A::add(txv, tyv), tzv));
            const R K = A::sub(A::mul(KA, lap), A::mul(KB, Pot::dV(f, cv, c0, q)));
            const KickOut<R> ko = kick_val<R>(piC[f][k], K, a.h1, a.h2);
            outp[f][k] = ko.next;
            if (RED & 1) site_pi2 = f == 0 ? ko.mid * ko.mid : site_pi2 + ko.mid * ko.mid;
          } else if (RED & 1) {
            const double pc = (double)piC[f][k];
            site_pi2 = f == 0 ? pc * pc : site_pi2 + pc * pc;
          }
          if ((RED & 2) && vk) {
            const R gx = A::sub(nxt[f][k], c), gy = A::sub(yp[f][k], c), gz = A::sub(zn, c);
            acc_g2 += (double)A::mul(A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz)), inv_dx2);
          }
        }
        if ((RED & 1) && vk) acc_pi2 += site_pi2;
        if ((RED & 2) && vk) acc_v += (double)Pot::V(cv, c0q, qh);
      }
      // stores: interior pair, then the periodic ghost copies of boundary sites
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        const long long o = (long long)f * pd.comp;
        if (DRIFT) {
          if (v0 && v1) {
            *reinterpret_cast<V2 *>(fout + o + base) = V2{outf[f][0], outf[f][1]};
          } else if (v0) {
            fout[o + base] = outf[f][0];
          }
        }
        if (KICK) {
          if (v0 && v1) {
            *reinterpret_cast<V2 *>(pout + o + base) = V2{outp[f][0], outp[f][1]};
          } else if (v0) {
            pout[o + base] = outp[f][0];
          }
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const bool vk = k == 0 ? v0 : v1;
          if (!vk) continue;
          const int zk = z + k;
          long long g[3];
          int ng = 0;
          if (y == 0) g[ng++] = pd.at(x, N, zk);
          if (y == N - 1) g[ng++] = pd.at(x, -1, zk);
          if (zk == 0) g[ng++] = pd.at(x, y, N);
          if (zk == N - 1 && ng < 3) g[ng++] = pd.at(x, y, -1);
          for (int i = 0; i < ng; ++i) {
            if (DRIFT) fout[o + g[i]] = outf[f][k];
            if (KICK) pout[o + g[i]] = outp[f][k];
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
        for (int k = 0; k < 2; ++k) {
          prev[f][k] = cur[f][k];
          cur[f][k] = nxt[f][k];
          if (LOADP) piC[f][k] = piN[f][k];
        }
    }
    if (RED) {
      double v[kRedSlots] = {acc_pi2, acc_g2, acc_v};
      block_reduce<kRedSlots, kSweepThreads>(v, red_smem);
      if (tid == 0) {
        const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
        for (int k = 0; k < kRedSlots; ++k) partials[bid * kRedSlots + k] = v[k];
      }
    }
    return;
  }

drain:
  // A wait gave up: flag it, then let thread 0 wait (bounded) for the copies still in flight so no
  // TMA write lands in shared memory after the block has left.
  if (tid == 0) {
    atomicOr(err, 1);
    for (int j = waited; j < issued; ++j) (void)mbar_wait(&bars[j % S], (uint32_t)((j / S) & 1), a.tries);
  }
}

// ---- padded elementwise / row kernels -------------------------------------------------------------
// Sum over interior sites of sum_f pi_f^2 into slot 0 of each block's partial row.
template <class R, int NS>
__global__ void __launch_bounds__(256) k_reduce_pi2_pad(const R *pi, Pad pd, double *__restrict__ partials)
{
  __shared__ double smem[(256 / 32) * kRedSlots];
  const int N = pd.N;
  double acc = 0;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int x = (int)(r / N), y = (int)(r % N);
    for (int z = threadIdx.x; z < N; z += blockDim.x) {
      const long long s = pd.at(x, y, z);
      double v = 0;
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        const double p = (double)pi[f * pd.comp + s];
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
    k_measure_pad(const R *fld, const R *pi, Pad pd, double inv_dx2d, double c0qd, double qhd, double am,
                  double *__restrict__ partials)
{
  using A = Ar<R>;
  using Pot = Lphi4<R, NS>;
  __shared__ double smem[(256 / 32) * kMeasSlots];
  const int N = pd.N;
  const R inv_dx2 = (R)inv_dx2d, c0q = (R)c0qd, qh = (R)qhd;
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
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        const long long o = f * pd.comp;
        const R c = fld[o + s];
        v[f] = c;
        const R gx = A::sub(fld[o + sx], c), gy = A::sub(fld[o + sy], c), gz = A::sub(fld[o + sz], c);
        const R g2 = A::mul(A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz)), inv_dx2);
        const double p = (double)pi[o + s];
        const double m = p * am;
        acc[6 * f + 0] += p * p;
        acc[6 * f + 1] += (double)g2;
        acc[6 * f + 2] += (double)c;
        acc[6 * f + 3] += (double)c * (double)c;
        acc[6 * f + 4] += m;
        acc[6 * f + 5] += m * m;
      }
#pragma unroll
      for (int k = 0; k < NS; ++k) acc[6 * NS + k] += (double)Pot::Vterm(k, v, c0q, qh);
    }
  }
  block_reduce<kMeasSlots, 256>(acc, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < kMeasSlots; ++k) partials[(size_t)blockIdx.x * kMeasSlots + k] = acc[k];
}

// Host-order planes (plane p = f N + x, N x N each) -> padded interior, with type conversion.
template <class S, class D>
__global__ void __launch_bounds__(256) k_scatter(const S *__restrict__ src, D *__restrict__ dst, Pad pd, long long p0, long long np)
{
  const int N = pd.N;
  for (long long r = blockIdx.x; r < np * N; r += gridDim.x) {
    const long long p = p0 + r / N;
    const int y = (int)(r % N);
    const int f = (int)(p / N), x = (int)(p % N);
    const long long o = (long long)f * pd.comp + pd.at(x, y, 0);
    for (int z = threadIdx.x; z < N; z += blockDim.x) dst[o + z] = (D)src[r * N + z];
  }
}

template <class S, class D>
__global__ void __launch_bounds__(256) k_gather(const S *__restrict__ src, D *__restrict__ dst, Pad pd, long long p0, long long np)
{
  const int N = pd.N;
  for (long long r = blockIdx.x; r < np * N; r += gridDim.x) {
    const long long p = p0 + r / N;
    const int y = (int)(r % N);
    const int f = (int)(p / N), x = (int)(p % N);
    const long long o = (long long)f * pd.comp + pd.at(x, y, 0);
    for (int z = threadIdx.x; z < N; z += blockDim.x) dst[r * N + z] = (D)src[o + z];
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
