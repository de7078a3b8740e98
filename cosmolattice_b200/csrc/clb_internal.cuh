// clb_internal.cuh - device-side state and helpers shared by the sm_100a kernels of libclb200.
#pragma once

#include <cstdlib>

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace clb {

// Number of reduction slots every sweep writes per block: <pi^2>, <grad^2>, <V>.
constexpr int kRedSlots = 3;
// Slots of the measurement reduction (per field: pi^2, grad^2, phi, phi^2, mom, mom^2; then V terms).
constexpr int kMeasSlots = 16;

// Scale-factor state, cached volume averages and the per-sweep coefficients, kept in device
// memory so a whole evolve() call runs without host round trips.  Field names follow
// ScaleFactorBase (abstractmodel/scalefactorbase.h:20-21) and ScalarBase (scalarbase.h).
struct DevState {
  double aI, aSI, aIM, aDotI, aDotSI, aDotSIM;
  double pi2AvI, pi2AvSI, pi2AvSIM, grad2AvI, potAvI, potAvSI;
  double grad2AvSI; // position Verlet: <grad^2> at the half step (positionverlet.h:258-266)
  // coefficients read by the sweeps
  double drift_p; // pow(aSI, alpha - 3) (velocityverlet.h:183); position Verlet pow(aI, alpha - 3)
                  // (positionverlet.h:172)
  double kick_A;  // pow(aI, 1 + alpha)               (scalarsingletkernels.h:266)
  double kick_B;  // pow(aI, 3 + alpha)
  int32_t status; // 0 ok, 1 non-finite average seen
  int32_t pad;
  // FP32/FP64-split storage: phi = ref_phi + s, pi = ref_pi + p with s, p the FP32 arrays and the
  // homogeneous references in FP64, advanced by the same VV map as a homogeneous site.  Two slots:
  // a sweep reads slot rs and its first block writes the advanced values into slot rs ^ 1.
  double ref_phi[2][2]; // [slot][field]
  double ref_pi[2][2];
};

// Constants of the scale-factor equation (scalefactorkernels.h:73-77) and Friedmann constraint.
struct SFParams {
  double alpha;
  double fm2;     // (fStar / MPl)^2
  double dt;
  double inv_n3;  // 1 / N^3
};

// Operations of the one-thread tail that follows a reducing sweep.  Applied in field order.
enum TailFlags : uint32_t {
  T_STORE_PI2_I = 1u << 0,  // pi2AvI = <pi^2>                         (velocityverlet.h:251)
  T_STORE_PI2_LF = 1u << 1, // pi2AvSIM = pi2AvSI; pi2AvSI = <pi^2>; pi2AvI = mean (leapfrog.h:241-245)
  T_STORE_FIELDS = 1u << 2, // grad2AvI = <grad^2>; potAvI = <V>       (velocityverlet.h:258-266)
  T_STORE_ALL = 1u << 3,    // Averages::setAllAverages                (averages.h:349-358)
  T_VV_KICK_ONE = 1u << 4,  // aDotI = aDotSI + dt/2 F w               (velocityverlet.h:171-174)
  T_VV_KICK_HALF = 1u << 5, // aDotSI = aDotI + dt/2 F w2              (velocityverlet.h:165-169)
  T_VV_DRIFT = 1u << 6,     // a drift with weight w2                  (velocityverlet.h:239-242)
  T_LF_KICK = 1u << 7,      // LeapFrog::kickScaleFactor               (leapfrog.h:124-129)
  T_LF_DRIFT = 1u << 8,     // LeapFrog::driftScaleFactor              (leapfrog.h:180-183)
  T_LF_SYNC = 1u << 9,      // aDotI = aDotSI + dt/2 F                 (leapfrog.h:111)
  T_LF_CTOR = 1u << 10,     // aDotSI = aDotI - dt/2 F                 (leapfrog.h:35)
  T_CORRECT_ADOT = 1u << 11,// aDotI = sqrt(Friedmann RHS)             (modelinitializer.h:77-78)
  T_HIST_EARLY = 1u << 12,  // history row right after the field averages (LF step end)
  T_STORE_PI2_B = 1u << 13, // a two-kick sweep's second momentum sums become the cached <pi^2>
                            // (after T_VV_KICK_HALF; the gauge sectors' tails)
  // PositionVerlet (positionverlet.h:45-99, 160-276), applied after the flags above, in this order:
  T_PV_STORE_SI = 1u << 14,  // grad2AvSI = <grad^2>; potAvSI = <V>      storeFieldsAveragesHalf (:258-266)
  T_PV_STORE_PI2 = 1u << 15, // pi2AvIM = pi2AvI; pi2AvI = <pi^2>; pi2AvSI = mean  storeMomentaAverages (:238-256)
  T_PV_KICK = 1u << 16,      // aDotI += dt getSI w                       kickScaleFactor (:160-163)
  T_PV_DRIFT_A2 = 1u << 17,  // aI += dt/2 aDotI w; aSI = (aIM + aI)/2    driftScaleFactorSecondHalf (:225-234)
  T_PV_DRIFT_A1 = 1u << 18,  // aIM = aI; aI += dt/2 aDotI w2; aSI = aI    driftScaleFactorFirstHalf (:209-222)
  T_PV_MODE = 1u << 19,      // drift coefficient pow(aI, alpha - 3), of the a before T_PV_DRIFT_A1
  // Fixed background (FixedBackgroundExpansion, fixedbackgroundexpansion.h:37-45): a and aDot are
  // the host's closed-form values fa, fb, applied after the flags above, in this order:
  T_FB_AIM = 1u << 20,       // aIM = aI
  T_FB_AI = 1u << 21,        // aI = fa
  T_FB_ASI = 1u << 22,       // aSI = fb                                 (leapfrog.h:171-175)
  T_FB_PV_HALF = 1u << 23,   // aIM = aI; aI = fb; aSI = aI              (positionverlet.h:209-216)
  T_FB_ADOT = 1u << 24       // aDotI = fb                               (sync: velocityverlet.h:121)
};

struct TailOp {
  uint32_t flags;
  int32_t nblocks; // number of partial rows to reduce (0: no reduction)
  double w;        // weight of T_VV_KICK_ONE
  double w2;       // weight of T_VV_KICK_HALF / T_VV_DRIFT
  double *hist;    // per-step history rows (kHistCols doubles), or null
  int64_t hist_row;// row written after this tail, -1 for none
  double fa, fb;   // fixed background: the values of T_FB_*
};

// Columns of the per-step history: a, aDot, <pi^2>, <grad^2>, <V> at the end of each step.
constexpr int kHistCols = 5;

// Per-launch geometry of the z-marching stencil sweeps.
struct SweepGeom {
  int N;
  int LX;         // x planes per block
  dim3 grid;
};

// Arithmetic with a pinned rounding sequence.  The FP64 form uses the _rn intrinsics so the
// compiler cannot contract a*b+c into an FMA: the FP64 path then rounds exactly where the
// reference's expression templates round, which the 1e-12 parity bar relies on.  The FP32 form
// lets the compiler fuse.
template <class R> struct Ar;
template <> struct Ar<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
};
template <> struct Ar<float> {
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
  static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
};

__device__ __forceinline__ double ipow_d(double x, int n)
{
  if (n == 0) return 1.0;
  if (n < 0) return 1.0 / ipow_d(x, -n);
  double r = x;
  for (int i = 1; i < n; ++i) r = __dmul_rn(r, x);
  return r;
}

// Programmatic dependent launch (sm_90+): griddep_wait blocks until the preceding kernel in the
// stream has completed and its writes are visible (a no-op when the launch has no programmatic
// dependency); griddep_launch lets the next kernel, if launched with the attribute, start its
// independent prologue once every block of this one has signalled or exited.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Deterministic block reduction of NV per-thread values; thread 0 of the block gets the sums.
template <int NV, int NT>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double *smem /* [NT/32][NV] */)
{
  const int lane = threadIdx.x & 31;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int warp = tid >> 5;
  // lanes are numbered along threadIdx.x first; blockDim.x is a multiple of 32 or the whole block
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    v[k] = s;
  }
  (void)lane;
  if ((tid & 31) == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) smem[warp * NV + k] = v[k];
  }
  __syncthreads();
  if (tid < 32) {
    constexpr int NW = NT / 32;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = tid < NW ? smem[tid * NV + k] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      v[k] = s;
    }
  }
}

// Periodic neighbour offsets of site s = (x N + y) N + z: op[d] to x + d, om[d] to x - d.
__device__ __forceinline__ void u1_offsets(int N, size_t s, long long (&op)[3], long long (&om)[3])
{
  const int z = (int)(s % (size_t)N);
  const size_t t = s / (size_t)N;
  const int y = (int)(t % (size_t)N);
  const int x = (int)(t / (size_t)N);
  const int c[3] = {x, y, z};
  const long long st[3] = {(long long)N * N, (long long)N, 1};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    op[d] = c[d] + 1 == N ? -(long long)(N - 1) * st[d] : st[d];
    om[d] = c[d] == 0 ? (long long)(N - 1) * st[d] : -st[d];
  }
}

// Site order of the gauge-model sweeps.
//   order 0: a grid-stride loop over s = (x N + y) N + z.
//   order 1 (bricks): the block's threads cover a 32 (z) x blockDim.x/32 (y) tile of one x-plane and
//     march it along x over runs of kBrickRun planes; the (tile, run) items go to the blocks in turn.
//     The plane a thread reads as its x + 1 neighbours is the plane of its next site, so those
//     values, and the y neighbours inside the tile, are re-read from L1 rather than from L2.
// Either order visits every site once; the per-site arithmetic is the same, and only the grouping
// of the volume sums into block partials differs.
constexpr int kBrickRun = 32;
// Bricks where they measured faster: lattices of at least 32 sites a side (a smaller one fills
// too little of a tile) and a sweep that gains from them (bricks = true; at 192^3 the lphi4SU2U1
// kicks 1.11x FP64 and 1.06x FP32, the FP32 lphi4U1 kick 1.04x, while the FP64 lphi4U1 kick lost
// 1.22x).  CLB_GAUGE_ORDER=0 or 1 forces the order.
inline int gauge_site_order(int N, bool bricks)
{
  if (const char *env = std::getenv("CLB_GAUGE_ORDER")) return std::atoi(env) != 0 ? 1 : 0;
  return bricks && N >= 32 ? 1 : 0;
}
template <class Fn> __device__ __forceinline__ void for_sites(int N, size_t n3, int order, Fn &&fn)
{
  if (order == 0) {
    for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) fn(s);
    return;
  }
  const int TY = (int)(blockDim.x >> 5);
  const int tz = (int)(threadIdx.x & 31), ty = (int)(threadIdx.x >> 5);
  const int ntz = (N + 31) >> 5, nty = (N + TY - 1) / TY, nxr = (N + kBrickRun - 1) / kBrickRun;
  const long long items = (long long)ntz * nty * nxr;
  const size_t plane = (size_t)N * N;
  for (long long it = blockIdx.x; it < items; it += gridDim.x) {
    const int zt = (int)(it % ntz);
    const long long r = it / ntz;
    const int yt = (int)(r % nty), xr = (int)(r / nty);
    const int z = zt * 32 + tz, y = yt * TY + ty;
    if (z >= N || y >= N) continue;
    const int xa = xr * kBrickRun, xb = min(N, xa + kBrickRun);
    size_t s = (size_t)xa * plane + (size_t)y * N + z;
    for (int x = xa; x < xb; ++x, s += plane) fn(s);
  }
}

// Asynchronous global -> shared copies (cp.async, sm_80+): 4, 8 or 16 bytes, both addresses
// aligned to the size.  A commit closes a group; wait_group<K> returns when at most K of this
// thread's groups are still in flight.
template <int B> __device__ __forceinline__ void cp_async(void *dst, const void *src)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (B == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

// VZ consecutive elements (VZ * sizeof(R) bytes, aligned to that size on both sides).
template <class R, int VZ> __device__ __forceinline__ void cp_run(R *dst, const R *src)
{
  constexpr int BYTES = VZ * (int)sizeof(R), CH = BYTES >= 16 ? 16 : BYTES;
#pragma unroll
  for (int o = 0; o < BYTES; o += CH)
    cp_async<CH>(reinterpret_cast<char *>(dst) + o, reinterpret_cast<const char *>(src) + o);
}

} // namespace clb
