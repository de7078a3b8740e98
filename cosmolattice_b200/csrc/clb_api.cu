// clb_api.cu - C ABI of libclb200: handle lifecycle, state transfer and the evolver schedules.
//
// The schedules restate the reference's composition loops:
//   VelocityVerlet::evolve   evolvers/velocityverlet.h:51-114
//   LeapFrog::evolve / sync  evolvers/leapfrog.h:42-116
// Everything between host calls runs on one CUDA stream with the scale factor kept on the
// device (DevState), so an evolve() of many steps issues kernels back to back with no host
// synchronisation until its end.

#include "../../include/clb200.h"
#include "clb_internal.cuh"
#include "clb_handle.cuh"
#include "clb_scalar.cuh"
#include "clb_spectrum.cuh"
#include "clb_sweep.cuh"
#include "clb_vv.h"

#include <cudaTypedefs.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace clb;

namespace {

thread_local std::string g_err;

constexpr int kElemBlocks = 148 * 8; // elementwise grid: 8 resident 256-thread blocks per SM
constexpr uint32_t kWaitTries = 1u << 24; // bound of each mbarrier wait in the sweeps
constexpr size_t kStageMin = (size_t)1 << 23; // host-transfer staging: >= 64 MiB of doubles
constexpr int kDefaultShapeFP64 = 0;          // ShapeW
constexpr int kDefaultShapeFP32 = 4;          // ShapeK
constexpr int kPlanesPerBlock = 32;           // x-run length of one sweep block

} // namespace

namespace clb {
// complex scalar + U(1) sector (clb_u1.cu)
int u1_create(clb_handle *h);
void u1_destroy(clb_handle *h);
int u1_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf);
int u1_get_state(clb_handle *h, double *fields, double *momenta, clb_scalefactor *sf);
int u1_initialize(clb_handle *h, int32_t correct_adot);
int u1_evolve(clb_handle *h, int64_t n);
int u1_sync(clb_handle *h);
int u1_measure(clb_handle *h, double e0, clb_measurement *m);
int u1_forward(clb_handle *h, int64_t nsteps, int32_t K, const double *w, int32_t nw, double *obs);
int u1_set_spectrum_seed(clb_handle *h, int which, int comp, const double *d_grad, double O, double abar);
int u1_backward(clb_handle *h, int32_t through_init, double *fields_bar, double *momenta_bar, clb_adjoint_grad *out);

// lphi4SU2U1 (clb_su2.cu)
int su2_create(clb_handle *h);
void su2_destroy(clb_handle *h);
int su2_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf);
int scalar_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf,
                     const double *means);
int su2_get_state(clb_handle *h, double *fields, double *momenta, clb_scalefactor *sf);
int su2_initialize(clb_handle *h, int32_t correct_adot);
int su2_evolve(clb_handle *h, int64_t n);
int su2_sync(clb_handle *h);
int su2_measure(clb_handle *h, double e0, clb_measurement *m);
int su2_tangent_begin(clb_handle *h, const double *couplings_dot, int32_t n, const double *fields_dot,
                      const double *momenta_dot, const clb_scalefactor *sf_dot);
int su2_tangent_get_state(clb_handle *h, double *fields_dot, double *momenta_dot, clb_scalefactor *sf_dot);
int su2_tangent_observable(clb_handle *h, const double *w, int32_t nw, double *obs, double *dobs);
int su2_tangent_end(clb_handle *h);
int su2_tangent_energies(clb_handle *h, double *E, double *dE);
const void *su2_tangent_component(clb_handle *h, int which, int comp, bool *f32, double *aI, double *daI);

const double *u1_component(clb_handle *h, int which, int comp, bool *gauge);
const double *su2_component(clb_handle *h, int which, int comp, bool *gauge);

// gravitational waves of the scalar singlets (clb_gws.cu)
void gw_kick_step(clb_handle *h);
void gw_drift(clb_handle *h);
void gw_sync(clb_handle *h);
void gw_set_synced(clb_handle *h, bool s);
void gw_destroy(clb_handle *h);

// Records a handle-less failure for clb_last_error(NULL); used by entry points in other units.
__attribute__((visibility("hidden"))) void set_global_error(const std::string &m) { g_err = m; }
} // namespace clb


namespace {


// Launch with the programmatic-stream-serialization attribute: the kernel may start while the
// previous kernel in the stream drains; it waits (griddep_wait) before touching dependent data.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args &&...args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// Sweep geometry: bz x by (z, y) sites per block; the x direction is split so the grid holds about
// two waves of resident blocks.
void setup_geometry(clb_handle *h, int blocks_per_sm)
{
  const int N = h->N;
  const int gx = (N + h->bz - 1) / h->bz, gy = (N + h->by - 1) / h->by;
  // Many short x-runs (about 32 planes) beat few long ones: a block's plane rate is bounded by its
  // own pipeline, so throughput comes from many blocks cycling through the SMs.  A small lattice
  // has few (z, y) tiles (64^3: 8), so its runs are shortened, down to one plane, until the grid
  // fills two waves of resident blocks (the extra halo planes then come from L2).
  int xs = std::max(1, (N + kPlanesPerBlock - 1) / kPlanesPerBlock);
  const int waves = 2 * 148 * std::max(1, blocks_per_sm);
  if ((long long)gx * gy * xs < waves) xs = std::max(xs, std::min(N, (waves + gx * gy - 1) / (gx * gy)));
  xs = std::max(1, std::min(xs, N));
  if (const char *env = std::getenv("CLB_SWEEP_XS")) xs = std::max(1, std::min(N, std::atoi(env)));
  int LX = (N + xs - 1) / xs;
  xs = (N + LX - 1) / LX;
  h->sa.LX = LX;
  h->sweep_grid = dim3(gx, gy, xs);
  h->sweep_blocks = gx * gy * xs;
}

template <class R> R *F(clb_handle *h, int b) { return static_cast<R *>(h->fld[b]); }
template <class R> R *P(clb_handle *h, int b) { return static_cast<R *>(h->pi[b]); }

// ---- kernel launchers (templated on storage type and field count) ----------------------------
template <class R, int NS, class SH, int DRIFT, bool KICK, int RED>
void sweep_sh(clb_handle *h, int kind, int fb, int pb, int fo, int po, double dtw, double h1, double h2,
              double dtw0 = 0.0)
{
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_sweep<R, NS, SH, DRIFT, KICK, RED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         160 * 1024);
    attr_set = true;
  }
  SweepArgs a = h->sw;
  a.dtw = dtw;
  a.h1 = h1;
  a.h2 = h2;
  a.dtw0 = dtw0;
  a.rs = h->rs;
  if (h->pdl_now)
    CLB_LAUNCH(h, kind,
               launch_pdl(k_sweep<R, NS, SH, DRIFT, KICK, RED>, h->sweep_grid, dim3(SH::TZ, SH::TY), h->sweep_smem,
                          h->stream, h->tm_f[fb], h->tm_p[pb], static_cast<R *>(h->fld[fo]), static_cast<R *>(h->pi[po]),
                          a, (const DevState *)h->d_st, h->d_part, h->d_err));
  else
    CLB_LAUNCH(h, kind,
               k_sweep<R, NS, SH, DRIFT, KICK, RED><<<h->sweep_grid, dim3(SH::TZ, SH::TY), h->sweep_smem, h->stream>>>(
                   h->tm_f[fb], h->tm_p[pb], static_cast<R *>(h->fld[fo]), static_cast<R *>(h->pi[po]), a, h->d_st,
                   h->d_part, h->d_err));
  if (sizeof(R) == 4 && (DRIFT || KICK)) h->rs ^= 1; // the launch advanced the FP64 references
}

template <class R, int NS, int DRIFT, bool KICK, int RED>
void sweep(clb_handle *h, int kind, int fb, int pb, int fo, int po, double dtw, double h1, double h2,
           double dtw0 = 0.0)
{
  if constexpr (NS == 1) {
    if (h->shape == 1) return sweep_sh<R, NS, ShapeQ, DRIFT, KICK, RED>(h, kind, fb, pb, fo, po, dtw, h1, h2, dtw0);
    if (h->shape == 2) return sweep_sh<R, NS, ShapeH, DRIFT, KICK, RED>(h, kind, fb, pb, fo, po, dtw, h1, h2, dtw0);
    if (h->shape == 3) return sweep_sh<R, NS, ShapeL, DRIFT, KICK, RED>(h, kind, fb, pb, fo, po, dtw, h1, h2, dtw0);
    if (h->shape == 4) return sweep_sh<R, NS, ShapeK, DRIFT, KICK, RED>(h, kind, fb, pb, fo, po, dtw, h1, h2, dtw0);
  }
  sweep_sh<R, NS, ShapeW, DRIFT, KICK, RED>(h, kind, fb, pb, fo, po, dtw, h1, h2, dtw0);
}

template <class R, int NS> struct Launch {
  // kick in place: pi += h K(phi)
  static void kick(clb_handle *h, double hk)
  {
    sweep<R, NS, false, true, 0>(h, K_KICK, h->cf, h->cp, h->cf, h->cp, 0.0, hk, 0.0);
  }
  // fused: drift (dtw) + kick (h1, h2) + averages, ping-pong buffers
  static void fused(clb_handle *h, double dtw, double h1, double h2, bool red)
  {
    const int nf = h->cf ^ 1, np = h->cp ^ 1;
    if (red)
      sweep<R, NS, true, true, 3>(h, K_FUSED, h->cf, h->cp, nf, np, dtw, h1, h2);
    else
      sweep<R, NS, true, true, 0>(h, K_FUSED, h->cf, h->cp, nf, np, dtw, h1, h2);
    h->cf = nf;
    h->cp = np;
  }
  // position-Verlet stage after the first: the previous stage's second drift (dtw0) and this
  // stage's first drift (dtw), each rounded as the reference's, kick (hk), averages
  static void fused_pv(clb_handle *h, double dtw0, double dtw, double hk, bool red)
  {
    const int nf = h->cf ^ 1, np = h->cp ^ 1;
    if (red)
      sweep<R, NS, 2, true, 3>(h, K_FUSED, h->cf, h->cp, nf, np, dtw, hk, 0.0, dtw0);
    else
      sweep<R, NS, 2, true, 0>(h, K_FUSED, h->cf, h->cp, nf, np, dtw, hk, 0.0, dtw0);
    h->cf = nf;
    h->cp = np;
  }
  // drift (dtw) with optional field averages, writes the other field buffer
  static void drift_fields(clb_handle *h, double dtw, bool red)
  {
    const int nf = h->cf ^ 1;
    if (red)
      sweep<R, NS, true, false, 2>(h, K_DRIFT_SWEEP, h->cf, h->cp, nf, h->cp, dtw, 0.0, 0.0);
    else
      sweep<R, NS, true, false, 0>(h, K_DRIFT_SWEEP, h->cf, h->cp, nf, h->cp, dtw, 0.0, 0.0);
    h->cf = nf;
  }
  // elementwise in-place drift over the whole padded arrays (ghosts stay periodic copies)
  static void drift(clb_handle *h, double dtw)
  {
    CLB_LAUNCH(h, K_DRIFT,
               k_drift<R><<<kElemBlocks, 256, 0, h->stream>>>(F<R>(h, h->cf), P<R>(h, h->cp),
                                                               (size_t)NS * (size_t)h->pd.comp, dtw, h->d_st, h->rs,
                                                               NS));
    if (sizeof(R) == 4) h->rs ^= 1;
  }
  // <pi^2> partials (elementwise grid)
  static int reduce_pi2(clb_handle *h)
  {
    CLB_LAUNCH(h, K_RED_PI2, k_reduce_pi2_pad<R, NS><<<kElemBlocks, 256, 0, h->stream>>>(P<R>(h, h->cp), h->pd, h->d_st, h->rs, h->d_part));
    return kElemBlocks;
  }
  // <grad^2>, <V> (and <pi^2> with all=true) partials (sweep grid)
  static int reduce_fields(clb_handle *h, bool all)
  {
    if (all)
      sweep<R, NS, false, false, 3>(h, K_RED_FIELDS, h->cf, h->cp, h->cf, h->cp, 0.0, 0.0, 0.0);
    else
      sweep<R, NS, false, false, 2>(h, K_RED_FIELDS, h->cf, h->cp, h->cf, h->cp, 0.0, 0.0, 0.0);
    return h->sweep_blocks;
  }
  static void measure(clb_handle *h, double am)
  {
    CLB_LAUNCH(h, K_MEASURE,
               k_measure_pad<R, NS><<<kElemBlocks, 256, 0, h->stream>>>(F<R>(h, h->cf), P<R>(h, h->cp), h->pd,
                                                                        h->sa.inv_dx2, h->sa.cs.mc, am, h->d_st,
                                                                        h->rs, h->d_part));
    CLB_LAUNCH(h, K_MEASURE, k_sum_partials<kMeasSlots><<<1, 256, 0, h->stream>>>(h->d_part, kElemBlocks, h->d_sums));
  }
};

// Host arrays (plane after plane, N x N each) <-> padded device components, through the staging
// buffer in whole planes, with FP32 conversion on the GPU and the periodic ghosts filled after upload.
cudaError_t upload(clb_handle *h, const double *src, void *dst, CompOffsets off)
{
  const long long planes = (long long)h->NS * h->N, per = (long long)h->N * h->N;
  const long long chunk = std::max<long long>(1, (long long)h->stage_n / per);
  for (long long p0 = 0; p0 < planes; p0 += chunk) {
    const long long np = std::min(chunk, planes - p0);
    cudaError_t r = cudaMemcpyAsync(h->d_stage, src + p0 * per, (size_t)(np * per) * sizeof(double),
                                    cudaMemcpyDefault, h->stream);
    if (r != cudaSuccess) return r;
    if (h->fp32)
      CLB_LAUNCH(h, K_CONVERT, k_scatter<double, float><<<kElemBlocks, 256, 0, h->stream>>>(
                                   h->d_stage, static_cast<float *>(dst), h->pd, p0, np, off));
    else
      CLB_LAUNCH(h, K_CONVERT, k_scatter<double, double><<<kElemBlocks, 256, 0, h->stream>>>(
                                   h->d_stage, static_cast<double *>(dst), h->pd, p0, np, off));
  }
  if (h->fp32)
    CLB_LAUNCH(h, K_CONVERT, k_fill_ghosts<float><<<kElemBlocks, 256, 0, h->stream>>>(static_cast<float *>(dst), h->pd, h->NS));
  else
    CLB_LAUNCH(h, K_CONVERT, k_fill_ghosts<double><<<kElemBlocks, 256, 0, h->stream>>>(static_cast<double *>(dst), h->pd, h->NS));
  return cudaGetLastError();
}

cudaError_t download(clb_handle *h, const void *src, double *dst, CompOffsets off)
{
  const long long planes = (long long)h->NS * h->N, per = (long long)h->N * h->N;
  const long long chunk = std::max<long long>(1, (long long)h->stage_n / per);
  for (long long p0 = 0; p0 < planes; p0 += chunk) {
    const long long np = std::min(chunk, planes - p0);
    if (h->fp32)
      CLB_LAUNCH(h, K_CONVERT, k_gather<float, double><<<kElemBlocks, 256, 0, h->stream>>>(
                                   static_cast<const float *>(src), h->d_stage, h->pd, p0, np, off));
    else
      CLB_LAUNCH(h, K_CONVERT, k_gather<double, double><<<kElemBlocks, 256, 0, h->stream>>>(
                                   static_cast<const double *>(src), h->d_stage, h->pd, p0, np, off));
    cudaError_t r = cudaMemcpyAsync(dst + p0 * per, h->d_stage, (size_t)(np * per) * sizeof(double),
                                    cudaMemcpyDeviceToHost, h->stream);
    if (r != cudaSuccess) return r;
  }
  return cudaStreamSynchronize(h->stream);
}

// 3-D tensor map over the stacked padded components: dims {Zp, Yp, NS N}, box = one plane tile.
bool encode_map(clb_handle *h, void *base, CUtensorMap *map, std::string &why)
{
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      why = "cuTensorMapEncodeTiled not available from the driver";
      return false;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const Pad &pd = h->pd;
  const cuuint64_t dims[3] = {(cuuint64_t)pd.Zp, (cuuint64_t)pd.Yp, (cuuint64_t)h->NS * (cuuint64_t)pd.N};
  const cuuint64_t strides[2] = {(cuuint64_t)pd.Zp * h->esz, (cuuint64_t)pd.plane * h->esz};
  const cuuint32_t boxz = (cuuint32_t)(h->bz + 2 * (16 / (int)h->esz));
  const cuuint32_t box[3] = {boxz, (cuuint32_t)(h->by + 2), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(map, h->fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims,
                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    why = "cuTensorMapEncodeTiled returned " + std::to_string((int)r);
    return false;
  }
  return true;
}

void tail(clb_handle *h, uint32_t flags, int nblocks, double w = 0, double w2 = 0, int64_t hist_row = -1,
          double fa = 0, double fb = 0)
{
  TailOp op{flags, nblocks, w, w2, hist_row >= 0 ? h->d_hist : nullptr, hist_row, fa, fb};
  if (h->pdl_now)
    CLB_LAUNCH(h, K_TAIL, launch_pdl(k_tail, dim3(1), dim3(kTailThreads), 0, h->stream, (const double *)h->d_part, op,
                                     h->d_st, h->sp));
  else
    CLB_LAUNCH(h, K_TAIL, k_tail<<<1, kTailThreads, 0, h->stream>>>(h->d_part, op, h->d_st, h->sp));
}

// Dispatch on (storage, field count).
template <template <class, int> class Fn, class... Args> void dispatch(clb_handle *h, Args... args)
{
  if (h->fp32) {
    if (h->NS == 1) Fn<float, 1>::run(h, args...);
    else Fn<float, 2>::run(h, args...);
  } else {
    if (h->NS == 1) Fn<double, 1>::run(h, args...);
    else Fn<double, 2>::run(h, args...);
  }
}

// ---- schedules --------------------------------------------------------------------------------
// VelocityVerlet::evolve, n steps (velocityverlet.h:51-114).
// Fixed-background tail: the flags' scale-factor values from the closed form (no reduction).
void fb_tail(clb_handle *h, uint32_t flags, double fa, double fb = 0.0)
{
  tail(h, flags, 0, 0, 0, -1, fa, fb);
}

template <class R, int NS> struct EvolveVV {
  static void run(clb_handle *h, int64_t nsteps)
  {
    using L = Launch<R, NS>;
    const double dt = h->cfg.dt;
    const bool ex = h->cfg.expansion != 0;
    const std::vector<double> &ws = h->ws;
    const size_t P = ws.size(), S = 2 * P - 1;
    auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
    if (h->fb) {
      // fixed background (velocityverlet.h:74-118, 225-231): no a-kicks and no averages; the
      // a-drift sets aI = a(t + w dt) and leaves aSI, which the field drift reads, as it was
      const double t0 = h->cfg.t0;
      if (h->cfg.path == CLB_PATH_REFERENCE) {
        for (int64_t s = 0; s < nsteps; ++s) {
          double tc = h->fb_t - t0;
          for (size_t i = 0; i < S; ++i) {
            const double w = wof(i);
            L::kick(h, w * dt / 2);
            fb_tail(h, T_FB_AIM | T_FB_AI, h->fb_a(tc + w * dt));
            L::drift(h, dt * w);
            L::kick(h, w * dt / 2);
            tc += dt * w;
          }
          h->fb_t += dt;
        }
        return;
      }
      // With GWs, as in the fused loop below: after a step's last sweep, the GW drift (the a_SI
      // that the fixed background leaves as it was) and the next step's GW kick (its a_I)
      const int64_t total = nsteps * (int64_t)S;
      if (h->gw) gw_kick_step(h);
      L::kick(h, wof(0) * dt / 2);
      h->pdl_now = h->pdl;
      double tc = h->fb_t - t0;
      for (int64_t k = 0; k < total; ++k) {
        const size_t i = (size_t)(k % (int64_t)S);
        const double w = wof(i);
        const bool more = k + 1 < total;
        const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
        fb_tail(h, T_FB_AIM | T_FB_AI, h->fb_a(tc + w * dt));
        L::fused(h, dt * w, w * dt / 2, more ? wn * dt / 2 : 0.0, false);
        if (h->gw && i + 1 == S) gw_drift(h);
        if (h->gw && i + 1 == S && more) gw_kick_step(h);
        tc += dt * w;
        if (i + 1 == S) {
          h->fb_t += dt;
          tc = h->fb_t - t0;
        }
      }
      h->pdl_now = false;
      return;
    }
    if (h->cfg.path == CLB_PATH_REFERENCE) {
      for (int64_t s = 0; s < nsteps; ++s)
        for (size_t i = 0; i < S; ++i) {
          const double w = wof(i);
          if (ex) tail(h, T_VV_KICK_HALF, 0, 0, w);            // kickScaleFactorHalf
          L::kick(h, w * dt / 2);                              // kickScalar
          if (ex) tail(h, T_STORE_PI2_I | T_VV_DRIFT, L::reduce_pi2(h), 0, w); // <pi^2>, driftScaleFactor
          L::drift(h, dt * w);                                 // driftScalar
          if (ex) tail(h, T_STORE_FIELDS, L::reduce_fields(h, false));         // storeFieldsAverages
          L::kick(h, w * dt / 2);                              // kickScalar
          if (ex) // <pi^2>, kickScaleFactorOne; the last stage closes step s
            tail(h, T_STORE_PI2_I | T_VV_KICK_ONE, L::reduce_pi2(h), w, 0, i + 1 == S ? s : -1);
        }
      return;
    }
    // Fused: the second kick of a stage and the first kick of the next one act with the same
    // kernel K(phi', a) (no field or a update in between), so one sweep drifts phi, forms
    // pi_mid = pi + h1 K and pi_next = pi_mid + h2 K, and reduces <pi_mid^2>, <grad^2>, <V>.
    // With GWs (evolver.h:102-124): a GW kick before each step at the step's fields and a_I, and
    // a GW drift after it with the a_SI of its last stage; both after the step's last sweep and
    // before the tail that moves a on to the next step's first stage.
    const int64_t total = nsteps * (int64_t)S;
    const double w0 = wof(0);
    if (h->gw) gw_kick_step(h);
    if (ex) tail(h, T_VV_KICK_HALF, 0, 0, w0); // kickScaleFactorHalf
    L::kick(h, w0 * dt / 2);                  // kickScalar with a(t) before the drift
    if (ex) tail(h, T_VV_DRIFT, 0, 0, w0);     // driftScaleFactor
    h->pdl_now = h->pdl; // the fused sweeps and their tails overlap their launches
    for (int64_t k = 0; k < total; ++k) {
      const size_t i = (size_t)(k % (int64_t)S);
      const double w = wof(i);
      const bool more = k + 1 < total;
      const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
      L::fused(h, dt * w, w * dt / 2, more ? wn * dt / 2 : 0.0, ex);
      if (h->gw && i + 1 == S) gw_drift(h);
      if (h->gw && i + 1 == S && more) gw_kick_step(h); // a_I of the step's end, before the tail drifts a
      if (ex) {
        uint32_t fl = T_STORE_PI2_I | T_STORE_FIELDS | T_VV_KICK_ONE;
        if (more) fl |= T_VV_KICK_HALF | T_VV_DRIFT;
        tail(h, fl, h->sweep_blocks, w, wn, i + 1 == S ? k / (int64_t)S : -1);
      }
    }
    h->pdl_now = false;
  }
};

// PositionVerlet::evolve, n steps (positionverlet.h:45-99).  A stage: drift(dt/2 w) at
// pow(aI, alpha - 3), the first a half-drift, the half-step field averages, kick(w dt) at the
// half-step a, the momentum averages, the a-kick (getSI), the second a half-drift, drift(dt/2 w) at
// the new a, the field averages.
template <class R, int NS> struct EvolvePV {
  static void run(clb_handle *h, int64_t nsteps)
  {
    using L = Launch<R, NS>;
    const double dt = h->cfg.dt;
    const bool ex = h->cfg.expansion != 0;
    const std::vector<double> &ws = h->ws;
    const size_t P = ws.size(), S = 2 * P - 1;
    auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
    if (nsteps <= 0) return;
    if (h->fb) {
      // fixed background (positionverlet.h:45-99, 207-235): a half-drifts from the closed form, no
      // a-kick and no averages
      const double t0 = h->cfg.t0;
      if (h->cfg.path == CLB_PATH_REFERENCE) {
        tail(h, T_PV_MODE, 0);
        for (int64_t s = 0; s < nsteps; ++s) {
          double tc = h->fb_t - t0;
          for (size_t i = 0; i < S; ++i) {
            const double w = wof(i);
            L::drift(h, dt / 2 * w);
            fb_tail(h, T_PV_MODE | T_FB_PV_HALF, 0.0, h->fb_a(tc + w * dt / 2.0));
            L::kick(h, w * dt);
            fb_tail(h, T_PV_MODE | T_FB_AI, h->fb_a(tc + w * dt));
            L::drift(h, dt / 2 * w);
            tc += dt * w;
          }
          h->fb_t += dt;
        }
        return;
      }
      // fused: every stage after the first of the call pairs the previous stage's second drift
      // with its own first drift; one drift sweep closes the call.  With GWs the steps run one per
      // call, the integer-time state between them being what the GW kick reads (evolver.h:102-124).
      if (h->gw && nsteps > 1) {
        for (int64_t s = 0; s < nsteps; ++s) run(h, 1);
        return;
      }
      if (h->gw) gw_kick_step(h);
      const int64_t total = nsteps * (int64_t)S;
      double tc = h->fb_t - t0;
      fb_tail(h, T_PV_MODE | T_FB_PV_HALF, 0.0, h->fb_a(tc + wof(0) * dt / 2.0));
      h->pdl_now = h->pdl;
      double wprev = 0.0;
      for (int64_t k = 0; k < total; ++k) {
        const size_t i = (size_t)(k % (int64_t)S);
        const double w = wof(i);
        if (k == 0)
          L::fused(h, dt / 2 * w, w * dt, 0.0, false);
        else
          L::fused_pv(h, dt / 2 * wprev, dt / 2 * w, w * dt, false);
        const double a_end = h->fb_a(tc + w * dt);
        tc += dt * w;
        if (i + 1 == S) {
          h->fb_t += dt;
          tc = h->fb_t - t0;
        }
        if (k + 1 < total) {
          const double wn = wof((size_t)((k + 1) % (int64_t)S));
          fb_tail(h, T_PV_MODE | T_FB_AI | T_FB_PV_HALF, a_end, h->fb_a(tc + wn * dt / 2.0));
        } else {
          fb_tail(h, T_PV_MODE | T_FB_AI, a_end);
        }
        wprev = w;
      }
      L::drift_fields(h, dt / 2 * wprev, false);
      if (h->gw) gw_drift(h);
      h->pdl_now = false;
      return;
    }
    if (h->cfg.path == CLB_PATH_REFERENCE) {
      tail(h, T_PV_MODE, 0); // the drift coefficient of the current a
      for (int64_t s = 0; s < nsteps; ++s)
        for (size_t i = 0; i < S; ++i) {
          const double w = wof(i);
          L::drift(h, dt / 2 * w); // driftScalar
          if (ex) tail(h, T_PV_MODE | T_PV_STORE_SI | T_PV_DRIFT_A1, L::reduce_fields(h, false), 0, w);
          L::kick(h, w * dt); // kickScalar
          if (ex) tail(h, T_PV_MODE | T_PV_STORE_PI2 | T_PV_KICK | T_PV_DRIFT_A2, L::reduce_pi2(h), w, 0);
          L::drift(h, dt / 2 * w);
          if (ex) tail(h, T_PV_MODE | T_STORE_FIELDS, L::reduce_fields(h, false), 0, 0, i + 1 == S ? s : -1);
        }
      return;
    }
    // Fused: one sweep per stage drifts (the previous stage's second drift and this stage's first,
    // which act with the same a and pi), kicks and reduces the half-step field averages and <pi^2>;
    // its tail books them, kicks a, finishes this stage's a-drift and starts the next one's.  Each
    // step ends with its own drift sweep, whose averages are the integer-time ones.
    // With GWs (evolver.h:102-124): the GW kick before each step (a_I before the step's first a
    // half-drift) and the GW drift after the step's closing drift sweep (its a_SI), both before the
    // tail that starts the next step's a half-drift.
    const double w0 = wof(0);
    if (h->gw) gw_kick_step(h);
    tail(h, T_PV_MODE | (ex ? T_PV_DRIFT_A1 : 0u), 0, 0, w0);
    h->pdl_now = h->pdl;
    for (int64_t s = 0; s < nsteps; ++s)
      for (size_t i = 0; i < S; ++i) {
        const double w = wof(i);
        const bool last = i + 1 == S;
        if (i == 0)
          L::fused(h, dt / 2 * w, w * dt, 0.0, ex);
        else
          L::fused_pv(h, dt / 2 * wof(i - 1), dt / 2 * w, w * dt, ex);
        if (ex) {
          uint32_t fl = T_PV_MODE | T_PV_STORE_SI | T_PV_STORE_PI2 | T_PV_KICK | T_PV_DRIFT_A2;
          if (!last) fl |= T_PV_DRIFT_A1;
          tail(h, fl, h->sweep_blocks, w, last ? 0.0 : wof(i + 1));
        }
        if (last) {
          L::drift_fields(h, dt / 2 * w, ex);
          if (h->gw) {
            gw_drift(h);
            if (s + 1 < nsteps) gw_kick_step(h);
          }
          if (ex) tail(h, T_PV_MODE | T_STORE_FIELDS | (s + 1 < nsteps ? T_PV_DRIFT_A1 : 0u), h->sweep_blocks, 0, w0, s);
        }
      }
    h->pdl_now = false;
  }
};

// LeapFrog::evolve, n steps (leapfrog.h:42-89).
template <class R, int NS> struct EvolveLF {
  static void run(clb_handle *h, int64_t nsteps)
  {
    using L = Launch<R, NS>;
    const double dt = h->cfg.dt;
    const bool ex = h->cfg.expansion != 0;
    if (nsteps <= 0) return;
    if (h->fb) {
      // fixed background (leapfrog.h:55-89, 168-184): aI = a(t + dt), aSI = a(t + dt/2)
      const double t0 = h->cfg.t0;
      auto a_drift = [&]() {
        const double tm = h->fb_t - t0;
        fb_tail(h, T_FB_AIM | T_FB_AI | T_FB_ASI, h->fb_a(tm + dt), h->fb_a(tm + dt / 2.0));
      };
      if (h->cfg.path == CLB_PATH_REFERENCE) {
        for (int64_t s = 0; s < nsteps; ++s) {
          L::kick(h, (h->synced ? 0.5 : 1.0) * dt);
          a_drift();
          L::drift(h, dt);
          h->fb_t += dt;
          h->synced = false;
        }
        return;
      }
      // GW hooks as in the self-consistent fused leapfrog below
      if (h->gw) gw_kick_step(h);
      L::kick(h, (h->synced ? 0.5 : 1.0) * dt);
      a_drift();
      for (int64_t s = 1; s < nsteps; ++s) {
        h->fb_t += dt;
        L::fused(h, dt, dt, 0.0, false);
        if (h->gw) {
          gw_drift(h);
          gw_kick_step(h);
        }
        a_drift();
      }
      L::drift_fields(h, dt, false);
      if (h->gw) gw_drift(h);
      h->fb_t += dt;
      h->synced = false;
      return;
    }
    if (h->cfg.path == CLB_PATH_REFERENCE) {
      for (int64_t s = 0; s < nsteps; ++s) {
        const double weight = h->synced ? 0.5 : 1.0;
        L::kick(h, weight * dt);
        if (ex) tail(h, T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, L::reduce_pi2(h));
        L::drift(h, dt);
        if (ex) tail(h, T_STORE_FIELDS | T_HIST_EARLY, L::reduce_fields(h, false), 0, 0, s);
        h->synced = false;
      }
      return;
    }
    // Fused: drift of step n and kick of step n+1 in one sweep; the sweep's reductions are the
    // field averages of phi_{n+1} and <pi_{n+3/2}^2>, which the tail books in LeapFrog order.
    // With GWs (evolver.h:102-124): the GW kick of step n+1 reads phi_{n+1} and a_I of step n+1,
    // and the GW drift of step n the a_SI of step n; both hold between the fused sweep and its
    // tail, which drifts a on.
    const double weight = h->synced ? 0.5 : 1.0;
    if (h->gw) gw_kick_step(h);
    L::kick(h, weight * dt);
    if (ex) tail(h, T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, L::reduce_pi2(h));
    for (int64_t s = 1; s < nsteps; ++s) {
      L::fused(h, dt, dt, 0.0, ex);
      if (h->gw) {
        gw_drift(h);
        gw_kick_step(h);
      }
      if (ex)
        tail(h, T_STORE_FIELDS | T_HIST_EARLY | T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, h->sweep_blocks, 0, 0, s - 1);
    }
    L::drift_fields(h, dt, ex);
    if (h->gw) gw_drift(h);
    if (ex) tail(h, T_STORE_FIELDS | T_HIST_EARLY, h->sweep_blocks, 0, 0, nsteps - 1);
    h->synced = false;
  }
};

template <class R, int NS> struct SyncLF {
  static void run(clb_handle *h)
  {
    using L = Launch<R, NS>;
    if (!h->synced) {
      L::kick(h, 0.5 * h->cfg.dt);
      if (h->cfg.expansion && !h->fb) tail(h, T_STORE_PI2_I | T_LF_SYNC, L::reduce_pi2(h));
    }
    h->synced = true;
  }
};

template <class R, int NS> struct Init {
  static void run(clb_handle *h, int correct)
  {
    using L = Launch<R, NS>;
    uint32_t fl = T_STORE_ALL;
    if (h->cfg.expansion && correct == 1 && !h->fb) fl |= T_CORRECT_ADOT; // modelinitializer.h:74-80
    if (h->cfg.expansion && h->cfg.evolver == CLB_LF && correct != CLB_INIT_RESTART) fl |= T_LF_CTOR;
    tail(h, fl, L::reduce_fields(h, true));
  }
};

template <class R, int NS> struct Measure {
  static void run(clb_handle *h, double am) { Launch<R, NS>::measure(h, am); }
};

int sync_and_check(clb_handle *h, const char *where)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  collect_profile(h);
  DevState s;
  e = cudaMemcpy(&s, h->d_st, sizeof(s), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  int terr = 0;
  e = cudaMemcpy(&terr, h->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  if (terr != 0) return h->fail(CLB_ETIMEOUT, std::string(where) + ": a sweep's bounded wait for its tile loads gave up");
  if (s.status != 0) return h->fail(CLB_ENONFINITE, std::string(where) + ": a volume average or a(t) is not finite");
  return CLB_OK;
}

} // namespace

extern "C" {

const char *clb_version(void) { return "clb200 0.1 (sm_100a)"; }

const char *clb_last_error(const clb_handle *h) { return h ? h->err.c_str() : g_err.c_str(); }

int clb_create(const clb_config *cfg, const clb_model_desc *md, clb_handle **out)
{
  if (!cfg || !md || !out) {
    g_err = "clb_create: null argument";
    return CLB_EINVAL;
  }
  *out = nullptr;
  const bool u1 = md->kind == CLB_MODEL_LPHI4U1;
  const bool su2 = md->kind == CLB_MODEL_LPHI4SU2U1;

  if (md->kind != CLB_MODEL_LPHI4 && !u1 && !su2) {
    g_err = "clb_create: unknown model kind";
    return CLB_EUNSUPPORTED;
  }
  if (!u1 && !su2 && (md->n_scalars < 1 || md->n_scalars > 2)) {
    g_err = "clb_create: lphi4 supports 1 or 2 scalar singlets";
    return CLB_EUNSUPPORTED;
  }
  if (cfg->N < 2 || cfg->N > 4096) {
    g_err = "clb_create: N must be in [2, 4096]";
    return CLB_EINVAL;
  }
  if (!(cfg->dx > 0) || !std::isfinite(cfg->dx)) {
    g_err = "clb_create: dx must be positive";
    return CLB_EINVAL;
  }
  if (cfg->dt == 0 || !std::isfinite(cfg->dt)) {
    g_err = "clb_create: dt cannot be zero, abort.";  // runparameters.h:191
    return CLB_EINVAL;
  }
  if (cfg->precision != CLB_PREC_FP64 && cfg->precision != CLB_PREC_FP32_SPLIT) {
    g_err = "clb_create: unknown precision";
    return CLB_EINVAL;
  }
  if (cfg->path != CLB_PATH_FUSED && cfg->path != CLB_PATH_REFERENCE) {
    g_err = "clb_create: unknown path";
    return CLB_EINVAL;
  }
  if (!(md->fStar > 0) || !(md->MPl > 0) || !(md->omegaStar > 0)) {
    g_err = "clb_create: fStar, omegaStar and MPl must be positive";
    return CLB_EINVAL;
  }
  const bool fb = cfg->expansion && cfg->fixed_background;
  if (fb && !(std::fabs(cfg->H0) > 1e-8)) { // runParameterTolerance (fixedbackgroundexpansion.h:28-31)
    g_err = "For models that do not involve cosmic defects, you need to specify a non-zero H0 to run a simulation with "
            "fixed background. If you want to disable expansion, please set expansion = false in the input file.";
    return CLB_EINVAL;
  }
  std::vector<double> ws;
  if (cfg->evolver != CLB_LF) {
    ws = is_pv(cfg->evolver) ? pv_coefficients(cfg->evolver) : vv_coefficients(cfg->evolver);
    if (ws.empty()) {
      g_err = "clb_create: The evolver type you specified was not implemented in the Evolver class";  // evolver.h:366-368
      return CLB_EUNSUPPORTED;
    }
  }
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) {
    g_err = std::string("clb_create: cudaSetDevice: ") + cudaGetErrorString(e);
    return CLB_ECUDA;
  }
  clb_handle *h = new clb_handle();
  h->cfg = *cfg;
  h->md = *md;
  h->N = cfg->N;
  h->n3 = (size_t)cfg->N * cfg->N * cfg->N;
  h->fb = fb;
  if (fb) { // pEoS, H0 (fixedbackgroundexpansion.h:21-26)
    h->fb_p = 2.0 / (3.0 * (1.0 + cfg->omega_eos) - 2.0 * md->alpha);
    h->fb_H0 = cfg->H0;
    h->fb_t = cfg->t0;
  }
  if (u1 || su2) {
    h->ws = ws;
    const int r = u1 ? u1_create(h) : su2_create(h);
    if (r != CLB_OK) {
      g_err = std::string("clb_create: device allocation failed: ") + cudaGetErrorString(cudaGetLastError());
      clb_destroy(h);
      return r;
    }
    *out = h;
    return CLB_OK;
  }
  h->NS = md->n_scalars;
  h->fp32 = cfg->precision == CLB_PREC_FP32_SPLIT;
  h->esz = h->fp32 ? sizeof(float) : sizeof(double);
  h->ws = ws;
  h->pd = make_pad(h->N, (int)h->esz);
  ScalarArgs &a = h->sa;
  a.N = h->N;
  a.inv_dx2 = 1.0 / (cfg->dx * cfg->dx);
  a.cs.mc = ScalarModel::couplings(md->couplings);
  // ring depth: as many plane stages as fit in ~48 KiB, at least 3 (planes x, x+1 and one in flight)
  // sweep shape: default per storage type and field count, CLB_SWEEP_SHAPE=0..4 overrides (one field)
  h->shape = (h->NS == 1) ? (h->fp32 ? kDefaultShapeFP32 : kDefaultShapeFP64) : 0;
  if (const char *env = std::getenv("CLB_SWEEP_SHAPE")) {
    const int v = std::atoi(env);
    if (h->NS == 1 && v >= 0 && v <= 4) h->shape = v;
  }
  {
    // sites per block along z and y of ShapeW, ShapeQ, ShapeH, ShapeL, ShapeK
    static const int kShapeBZ[5] = {64, 64, 64, 128, 128};
    static const int kShapeBY[5] = {8, 16, 8, 8, 4};
    h->bz = kShapeBZ[h->shape];
    h->by = kShapeBY[h->shape];
  }
  if (const char *env = std::getenv("CLB_PDL")) h->pdl = std::atoi(env) != 0;
  const size_t box_bytes = (size_t)(h->bz + 2 * (16 / (int)h->esz)) * (size_t)(h->by + 2) * h->esz;
  const size_t slot = ((box_bytes + 127) / 128) * 128;
  const size_t stage_bytes = (size_t)h->NS * 2 * slot;
  size_t ring_budget = 32 * 1024;
  if (const char *env = std::getenv("CLB_SWEEP_RING_KB")) ring_budget = (size_t)std::max(8, std::atoi(env)) * 1024;
  h->S = (int)std::max<size_t>(3, std::min<size_t>(8, ring_budget / stage_bytes));
  h->sweep_smem = (size_t)h->S * stage_bytes + (size_t)h->S * sizeof(uint64_t) + 8 * kRedSlots * sizeof(double);
  const int bpsm = (int)std::max<size_t>(1, std::min<size_t>(8, (220 * 1024) / (h->sweep_smem + 1024)));
  setup_geometry(h, bpsm);
  SweepArgs &w = h->sw;
  w.pd = h->pd;
  w.LX = a.LX;
  w.S = h->S;
  w.tries = kWaitTries;
  // Lowers the bound of the sweeps' tile-load waits, so a test can make a wait run out and check
  // that the call reports CLB_ETIMEOUT (0: every wait gives up at once).
  if (const char *env = std::getenv("CLB_WAIT_TRIES")) w.tries = (uint32_t)std::strtoul(env, nullptr, 10);
  w.inv_dx2 = a.inv_dx2;
  w.cs = a.cs;
  const double fm = md->fStar / md->MPl;
  h->sp = SFParams{md->alpha, fm * fm, cfg->dt, 1.0 / (double)h->n3};
  h->part_rows = (size_t)std::max(h->sweep_blocks, kElemBlocks);
  const size_t bytes = (size_t)h->NS * (size_t)h->pd.comp * h->esz;
  const size_t nbuf = cfg->path == CLB_PATH_FUSED ? 2 : 1;
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  for (size_t b = 0; ok && b < nbuf; ++b) {
    ok = cudaMalloc(&h->fld[b], bytes) == cudaSuccess && cudaMalloc(&h->pi[b], bytes) == cudaSuccess;
    if (ok) ok = cudaMemset(h->fld[b], 0, bytes) == cudaSuccess && cudaMemset(h->pi[b], 0, bytes) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&h->d_st, sizeof(DevState)) == cudaSuccess;
  ok = ok && cudaMalloc(&h->d_part, h->part_rows * kMeasSlots * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&h->d_sums, kMeasSlots * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&h->d_err, sizeof(int)) == cudaSuccess && cudaMemset(h->d_err, 0, sizeof(int)) == cudaSuccess;
  ok = ok && cudaEventCreate(&h->ev_call[0]) == cudaSuccess && cudaEventCreate(&h->ev_call[1]) == cudaSuccess;
  if (ok) {
    h->stage_n = std::max<size_t>(kStageMin, (size_t)h->N * h->N);
    ok = cudaMalloc(&h->d_stage, h->stage_n * sizeof(double)) == cudaSuccess;
  }
  if (!ok) {
    g_err = std::string("clb_create: device allocation failed: ") + cudaGetErrorString(cudaGetLastError());
    clb_destroy(h);
    return CLB_ENOMEM;
  }
  for (size_t b = 0; b < nbuf; ++b) {
    std::string why;
    if (!encode_map(h, h->fld[b], &h->tm_f[b], why) || !encode_map(h, h->pi[b], &h->tm_p[b], why)) {
      g_err = "clb_create: tensor map: " + why;
      clb_destroy(h);
      return CLB_ECUDA;
    }
  }
  if (nbuf == 1) {
    h->tm_f[1] = h->tm_f[0];
    h->tm_p[1] = h->tm_p[0];
  }
  DevState s{};
  s.aI = s.aSI = s.aIM = 1.0;
  s.drift_p = s.kick_A = s.kick_B = 1.0;
  cudaMemcpy(h->d_st, &s, sizeof(s), cudaMemcpyHostToDevice);
  *out = h;
  return CLB_OK;
}

void clb_destroy(clb_handle *h)
{
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  u1_destroy(h);
  su2_destroy(h);
  gw_destroy(h);
  for (int b = 0; b < 2; ++b) {
    if (h->fld[b]) cudaFree(h->fld[b]);
    if (h->pi[b]) cudaFree(h->pi[b]);
  }
  if (h->d_st) cudaFree(h->d_st);
  if (h->d_part) cudaFree(h->d_part);
  if (h->d_sums) cudaFree(h->d_sums);
  if (h->d_err) cudaFree(h->d_err);
  if (h->d_hist) cudaFree(h->d_hist);
  if (h->d_stage) cudaFree(h->d_stage);
  if (h->plan_ok) cufftDestroy(h->plan);
  if (h->d_spec) cudaFree(h->d_spec);
  if (h->d_spec2) cudaFree(h->d_spec2);
  if (h->plan_inv_ok) cufftDestroy(h->plan_inv);
  if (h->d_spec_part) cudaFree(h->d_spec_part);
  if (h->d_spec_cnt) cudaFree(h->d_spec_cnt);
  if (h->d_spec_out) cudaFree(h->d_spec_out);
  if (h->d_spec_outc) cudaFree(h->d_spec_outc);
  for (auto &p : h->pend) {
    h->ev_pool.push_back(p.a);
    h->ev_pool.push_back(p.b);
  }
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  for (auto e : h->ev_call)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int clb_num_components(const clb_handle *h, int32_t *nf, int32_t *np)
{
  if (!h) return CLB_EINVAL;
  if (nf) *nf = h->NS;
  if (np) *np = h->su2 ? 19 : h->NS;
  return CLB_OK;
}

int clb_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf)
{
  if (!h || !fields || !momenta) return h ? h->fail(CLB_EINVAL, "clb_set_state: null argument") : CLB_EINVAL;
  if (h->u1) return u1_set_state(h, fields, momenta, sf);
  if (h->su2) return su2_set_state(h, fields, momenta, sf);
  return scalar_set_state(h, fields, momenta, sf, nullptr);
}

} // extern "C"

// lphi4 clb_set_state from host or device arrays; means (fields then momenta, one per scalar) are
// the FP32 split form's references, computed here from host arrays when null.
__attribute__((visibility("hidden"))) int clb::scalar_set_state(clb_handle *h, const double *fields, const double *momenta,
                                                                const clb_scalefactor *sf, const double *means)
{
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_set_state");
  h->cf = h->cp = 0;
  h->rs = 0;
  // FP32 split storage: each component is stored as its deviation from its FP64 volume mean
  CompOffsets fo{{0.0, 0.0}}, po{{0.0, 0.0}};
  if (h->fp32 && means) {
    for (int f = 0; f < h->NS; ++f) {
      fo.v[f] = means[f];
      po.v[f] = means[2 + f];
    }
  } else if (h->fp32) {
    for (int f = 0; f < h->NS; ++f) {
      double sf_ = 0, sp_ = 0;
      const double *fa = fields + (size_t)f * h->n3, *pa = momenta + (size_t)f * h->n3;
      for (size_t i = 0; i < h->n3; ++i) {
        sf_ += fa[i];
        sp_ += pa[i];
      }
      fo.v[f] = sf_ / (double)h->n3;
      po.v[f] = sp_ / (double)h->n3;
    }
  }
  e = upload(h, fields, h->fld[0], fo);
  if (e == cudaSuccess) e = upload(h, momenta, h->pi[0], po);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_set_state");
  DevState s{};
  s.aI = s.aSI = s.aIM = 1.0;
  if (sf) {
    s.aI = sf->aI;
    s.aSI = sf->aSI;
    s.aIM = sf->aIM;
    s.aDotI = sf->aDotI;
    s.aDotSI = sf->aDotSI;
    s.aDotSIM = sf->aDotSIM;
  }
  const double al = h->md.alpha;
  s.drift_p = std::pow(s.aSI, al - 3);
  s.kick_A = std::pow(s.aI, 1 + al);
  s.kick_B = std::pow(s.aI, 3 + al);
  for (int f = 0; f < 2; ++f) {
    s.ref_phi[0][f] = s.ref_phi[1][f] = fo.v[f];
    s.ref_pi[0][f] = s.ref_pi[1][f] = po.v[f];
  }
  e = cudaMemcpy(h->d_st, &s, sizeof(s), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_set_state");
  h->has_state = true;
  h->initialized = false;
  h->synced = true;
  return CLB_OK;
}

extern "C" {

int clb_get_state(clb_handle *h, double *fields, double *momenta, clb_scalefactor *sf)
{
  if (!h) return CLB_EINVAL;
  if (h->u1) return u1_get_state(h, fields, momenta, sf);
  if (h->su2) return su2_get_state(h, fields, momenta, sf);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_get_state");
  DevState cur;
  e = cudaMemcpy(&cur, h->d_st, sizeof(cur), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_get_state");
  CompOffsets fo{{0.0, 0.0}}, po{{0.0, 0.0}};
  if (h->fp32)
    for (int f = 0; f < h->NS; ++f) {
      fo.v[f] = cur.ref_phi[h->rs][f];
      po.v[f] = cur.ref_pi[h->rs][f];
    }
  auto fetch = [&](void *src, double *dst, CompOffsets off) -> cudaError_t {
    return dst ? download(h, src, dst, off) : cudaSuccess;
  };
  e = fetch(h->fld[h->cf], fields, fo);
  if (e == cudaSuccess) e = fetch(h->pi[h->cp], momenta, po);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_get_state");
  if (sf) {
    DevState s;
    e = cudaMemcpy(&s, h->d_st, sizeof(s), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return h->cuda_fail(e, "clb_get_state");
    sf->aI = s.aI;
    sf->aSI = s.aSI;
    sf->aIM = s.aIM;
    sf->aDotI = s.aDotI;
    sf->aDotSI = s.aDotSI;
    sf->aDotSIM = s.aDotSIM;
  }
  return CLB_OK;
}

int clb_initialize(clb_handle *h, int32_t correct_adot)
{
  if (!h) return CLB_EINVAL;
  if (!h->has_state) return h->fail(CLB_ESTATE, "clb_initialize: no state uploaded");
  h->fb_t = h->cfg.t0;
  if (correct_adot < 0 || correct_adot > CLB_INIT_RESTART)
    return h->fail(CLB_EINVAL, "clb_initialize: mode must be 0, 1 or CLB_INIT_RESTART");
  if (correct_adot == CLB_INIT_RESTART && h->fb)
    return h->fail(CLB_EUNSUPPORTED, "clb_initialize: a restart with a fixed background is not supported");
  if (h->u1 || h->su2) {
    const int r = h->u1 ? u1_initialize(h, correct_adot) : su2_initialize(h, correct_adot);
    if (r == CLB_OK) h->initialized = true;
    if (h->gw) gw_set_synced(h, correct_adot != CLB_INIT_RESTART); // evolver.h:52
    return r;
  }
  if (correct_adot == CLB_INIT_RESTART && h->fb)
    return h->fail(CLB_EUNSUPPORTED, "clb_initialize: a restart with a fixed background is not supported");
  dispatch<Init>(h, (int)correct_adot);
  h->synced = !(correct_adot == CLB_INIT_RESTART && h->cfg.evolver == CLB_LF); // leapfrog.h:30-31
  if (h->gw) gw_set_synced(h, correct_adot != CLB_INIT_RESTART);           // evolver.h:52
  h->fb_t = h->cfg.t0;
  int r = sync_and_check(h, "clb_initialize");
  if (r == CLB_OK) h->initialized = true;
  return r;
}

int clb_evolve(clb_handle *h, int64_t n)
{
  if (!h) return CLB_EINVAL;
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_evolve: call clb_initialize first");
  if (n < 0) return h->fail(CLB_EINVAL, "clb_evolve: negative step count");
  if (n == 0) return CLB_OK;
  h->hist_rows = 0;
  // a fixed background writes no history rows (a(t) is closed-form), so it needs no buffer
  if (h->cfg.expansion && !h->fb && n > h->hist_cap) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess && h->d_hist) e = cudaFree(h->d_hist);
    h->d_hist = nullptr;
    h->hist_cap = 0;
    if (e == cudaSuccess) e = cudaMalloc(&h->d_hist, (size_t)n * kHistCols * sizeof(double));
    if (e != cudaSuccess) return h->fail(CLB_ENOMEM, std::string("clb_evolve: history buffer: ") + cudaGetErrorString(e));
    h->hist_cap = n;
  }
  if (h->u1 || h->su2) {
    const int r = h->u1 ? u1_evolve(h, n) : su2_evolve(h, n);
    if (r == CLB_OK && h->cfg.expansion && !h->fb) h->hist_rows = n;
    return r;
  }
  cudaEventRecord(h->ev_call[0], h->stream);
  if (h->cfg.evolver == CLB_LF)
    dispatch<EvolveLF>(h, n);
  else if (is_pv(h->cfg.evolver))
    dispatch<EvolvePV>(h, n);
  else
    dispatch<EvolveVV>(h, n);
  cudaEventRecord(h->ev_call[1], h->stream);
  int r = sync_and_check(h, "clb_evolve");
  float ms = 0;
  if (cudaEventElapsedTime(&ms, h->ev_call[0], h->ev_call[1]) == cudaSuccess) h->last_evolve_ms = ms;
  if (r == CLB_OK && h->cfg.expansion && !h->fb) h->hist_rows = n;
  return r;
}

int clb_history(clb_handle *h, double *out, int64_t max_rows, int64_t *n_rows)
{
  if (!h || !n_rows) return h ? h->fail(CLB_EINVAL, "clb_history: null argument") : CLB_EINVAL;
  const int64_t n = std::min(max_rows, h->hist_rows);
  *n_rows = h->hist_rows;
  if (n > 0 && out) {
    cudaError_t e = cudaMemcpyAsync(out, h->d_hist, (size_t)n * kHistCols * sizeof(double), cudaMemcpyDeviceToHost,
                                    h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "clb_history");
  }
  return CLB_OK;
}

int clb_set_profiling(clb_handle *h, int32_t on)
{
  if (!h) return CLB_EINVAL;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_set_profiling");
  collect_profile(h);
  h->prof = on != 0;
  return CLB_OK;
}

int clb_reset_stats(clb_handle *h)
{
  if (!h) return CLB_EINVAL;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_reset_stats");
  collect_profile(h);
  for (int k = 0; k < 16; ++k) {
    h->launches[k] = 0;
    h->timed[k] = 0;
    h->kernel_ms[k] = 0;
  }
  return CLB_OK;
}

int clb_kernel_stats(clb_handle *h, clb_kernel_stat *out, int32_t max, int32_t *n)
{
  if (!h || !n) return h ? h->fail(CLB_EINVAL, "clb_kernel_stats: null argument") : CLB_EINVAL;
  *n = K_NKINDS;
  for (int k = 0; k < K_NKINDS && k < max && out; ++k) {
    std::memset(&out[k], 0, sizeof(out[k]));
    std::strncpy(out[k].name, kKindNames[k], sizeof(out[k].name) - 1);
    out[k].launches = h->launches[k];
    out[k].timed_launches = h->timed[k];
    out[k].total_ms = h->kernel_ms[k];
  }
  return CLB_OK;
}

int clb_last_evolve_ms(clb_handle *h, double *ms)
{
  if (!h || !ms) return CLB_EINVAL;
  *ms = h->last_evolve_ms;
  return CLB_OK;
}

void *clb_cuda_stream(clb_handle *h) { return h ? (void *)h->stream : nullptr; }

int clb_sync(clb_handle *h)
{
  if (!h) return CLB_EINVAL;
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_sync: call clb_initialize first");
  if (h->u1) return u1_sync(h);
  if (h->su2) return su2_sync(h);
  if (h->gw) gw_sync(h); // evolver.h:134-137, before the matter sync
  if (h->cfg.evolver == CLB_LF) dispatch<SyncLF>(h);
  if (h->fb) fb_tail(h, T_FB_ADOT, 0.0, h->fb_adot(h->fb_t - h->cfg.t0));
  return sync_and_check(h, "clb_sync");
}

int clb_measure(clb_handle *h, double e0, clb_measurement *m)
{
  if (!h || !m) return h ? h->fail(CLB_EINVAL, "clb_measure: null argument") : CLB_EINVAL;
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_measure: call clb_initialize first");
  if (h->u1) return u1_measure(h, e0, m);
  if (h->su2) return su2_measure(h, e0, m);
  DevState s;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&s, h->d_st, sizeof(s), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  const double al = h->md.alpha;
  const double am = std::pow(s.aI, al - 3);
  dispatch<Measure>(h, am);
  double sums[kMeasSlots];
  e = cudaMemcpyAsync(sums, h->d_sums, sizeof(sums), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  std::memset(m, 0, sizeof(*m));
  const double inv = 1.0 / (double)h->n3;
  auto ipow = [](double x, int n) {
    double r = x;
    for (int i = 1; i < n; ++i) r = r * x;
    return r;
  };
  const double am6 = 1.0 / ipow(s.aI, 6), am2 = 1.0 / ipow(s.aI, 2);
  const int NS = h->NS;
  double Etot = 0, pi2 = 0, g2 = 0, pot = 0;
  int k = 0;
  for (int f = 0; f < NS; ++f) {
    // EnergiesMeasurer::measure (energiesmeasurer.h:56-59)
    const double Ekin = 0.5 * (sums[6 * f + 0] * inv) * am6;
    const double Egrad = 0.5 * (sums[6 * f + 1] * inv) * am2;
    m->energies[k++] = Ekin;
    m->energies[k++] = Egrad;
    Etot += Ekin + Egrad;
    pi2 += sums[6 * f + 0];
    g2 += sums[6 * f + 1];
  }
  for (int t = 0; t < NS; ++t) {
    const double v = sums[6 * NS + t] * inv;
    m->energies[k++] = v;
    Etot += v;
    pot += sums[6 * NS + t];
  }
  m->energies[k++] = Etot;
  m->n_energies = k;
  if (h->cfg.expansion) {
    // HubbleConstraint::get -> Energies::rho -> Averages::setAllAverages (energies.h:219): the
    // cached averages are refreshed as a side effect, which later LF steps observe.
    s.potAvI = pot * inv;
    s.potAvSI = s.potAvI;
    s.pi2AvI = pi2 * inv;
    s.pi2AvSI = s.pi2AvI;
    s.grad2AvI = g2 * inv;
    const double rho = (0.5 * s.pi2AvI * am6 + 0.5 * s.grad2AvI * am2) + s.potAvI;
    const double LHS = s.aDotI * s.aDotI;
    const double RHS = std::pow(s.aI, 2 * al + 2) / 3. * h->sp.fm2 * rho;
    m->friedmann[0] = (LHS - RHS) / (LHS + RHS);
    m->friedmann[1] = LHS;
    m->friedmann[2] = RHS;
    e = cudaMemcpy(h->d_st, &s, sizeof(s), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  } else {
    m->friedmann[0] = std::fabs(1.0 - Etot / e0);
  }
  for (int f = 0; f < NS; ++f) {
    // MeansMeasurer::measure (meansmeasurer.h:28-48)
    const double phi = sums[6 * f + 2] * inv, phi2 = sums[6 * f + 3] * inv;
    const double mom = sums[6 * f + 4] * inv, mom2 = sums[6 * f + 5] * inv;
    const double r1 = phi2 - phi * phi, r2 = mom2 - mom * mom;
    m->means[f][0] = phi;
    m->means[f][1] = mom;
    m->means[f][2] = phi2;
    m->means[f][3] = mom2;
    m->means[f][4] = r1 > 0 ? std::sqrt(r1) : 0;
    m->means[f][5] = r2 > 0 ? std::sqrt(r2) : 0;
  }
  m->n_means = NS;
  m->aI = s.aI;
  m->aDotI = s.aDotI;
  m->hubble = s.aDotI / s.aI;
  return CLB_OK;
}

int clb_forward(clb_handle *h, int64_t nsteps, int32_t checkpoint_every, const double *weights, int32_t n_weights,
                double *observable)
{
  if (!h) return CLB_EINVAL;
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_forward: call clb_initialize first");
  if (!h->u1) return h->fail(CLB_EUNSUPPORTED, "clb_forward: the adjoint pair covers lphi4U1");
  return u1_forward(h, nsteps, checkpoint_every, weights, n_weights, observable);
}

int clb_backward(clb_handle *h, int32_t through_init, double *fields_bar, double *momenta_bar, clb_adjoint_grad *grad)
{
  if (!h) return CLB_EINVAL;
  if (!h->u1) return h->fail(CLB_EUNSUPPORTED, "clb_backward: the adjoint pair covers lphi4U1");
  return u1_backward(h, through_init, fields_bar, momenta_bar, grad);
}

int clb_tangent_begin(clb_handle *h, const double *couplings_dot, int32_t n_couplings, const double *fields_dot,
                      const double *momenta_dot, const clb_scalefactor *sf_dot)
{
  if (!h) return CLB_EINVAL;
  if (!h->su2) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_begin: the tangent-linear form covers lphi4SU2U1");
  if (!h->has_state) return h->fail(CLB_ESTATE, "clb_tangent_begin: call clb_set_state first");
  return su2_tangent_begin(h, couplings_dot, n_couplings, fields_dot, momenta_dot, sf_dot);
}

int clb_tangent_get_state(clb_handle *h, double *fields_dot, double *momenta_dot, clb_scalefactor *sf_dot)
{
  if (!h) return CLB_EINVAL;
  if (!h->su2) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_get_state: the tangent-linear form covers lphi4SU2U1");
  return su2_tangent_get_state(h, fields_dot, momenta_dot, sf_dot);
}

int clb_tangent_observable(clb_handle *h, const double *weights, int32_t n_weights, double *observable,
                           double *d_observable)
{
  if (!h) return CLB_EINVAL;
  if (!h->su2) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_observable: the tangent-linear form covers lphi4SU2U1");
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_tangent_observable: call clb_initialize first");
  return su2_tangent_observable(h, weights, n_weights, observable, d_observable);
}

int clb_tangent_energies(clb_handle *h, double *energies, double *d_energies)
{
  if (!h) return CLB_EINVAL;
  if (!h->su2) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_energies: the tangent-linear form covers lphi4SU2U1");
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_tangent_energies: call clb_initialize first");
  return su2_tangent_energies(h, energies, d_energies);
}

int clb_tangent_end(clb_handle *h)
{
  if (!h) return CLB_EINVAL;
  if (!h->su2) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_end: the tangent-linear form covers lphi4SU2U1");
  return su2_tangent_end(h);
}

constexpr int kSpecBlocks = 148 * 2;

} // extern "C"

namespace {

// PowerSpectrumMeasurer::powerSpectrum normalisation (powerspectrum.h:95-106) of a bin's sum of
// |f_k|^2 (linear in sum), and the bin's wave number ntil (in units of kIR).
double spec_value(const clb_handle *h, int ps_type, int ps_version, double dk, int b, unsigned long long c,
                  double nsum, double sum, double *ntil_out)
{
  const double pi = 3.14159265358979323846;
  const int N = h->N;
  const double dx = h->cfg.dx;
  const double kIR = 2 * pi / (N * dx);
  double N5 = 1;
  for (int i = 0; i < 5; ++i) N5 *= (double)N;
  const double ntil = (ps_version == 1 && c > 0) ? nsum / (double)c : (b + 0.5) * dk;
  *ntil_out = ntil;
  if (c == 0) return 0.0;
  if (ps_type == 1) return kIR * ntil * dx / dk / N5 / 2.0 / pi * sum;
  const double t = kIR * ntil * dx / N;
  return t * t * t / dk / 2.0 / (pi * pi) * (sum / (double)c);
}

// clb_spectrum, also returning the raw bin sums [sum |f|^2 | sum |n|] and counts, and whether the
// component belongs to a gauge field.
int spectrum_impl(clb_handle *h, int32_t which, int32_t comp, int32_t ps_type, int32_t ps_version, double dk,
                  int32_t nbins, int32_t fold, double *k_out, double *value_out, int64_t *count_out,
                  std::vector<double> &sums, std::vector<unsigned long long> &cnt, bool &gauge_comp_out)
{
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_spectrum: call clb_initialize first");
  const bool gauge_model = h->u1 || h->su2;
  bool gauge_comp = false;
  const double *plain = nullptr;
  if (gauge_model) {
    if (which < 0 || which > 1) return h->fail(CLB_EINVAL, "clb_spectrum: which must be 0 (field) or 1 (momentum)");
    plain = h->u1 ? u1_component(h, which, comp, &gauge_comp) : su2_component(h, which, comp, &gauge_comp);
    if (!plain) return h->fail(CLB_EINVAL, "clb_spectrum: component index out of range");
  }
  if (!gauge_model && (which < 0 || which > 1 || comp < 0 || comp >= h->NS))
    return h->fail(CLB_EINVAL, "clb_spectrum: which must be 0 (field) or 1 (momentum) and comp a scalar index");
  if (ps_type < 1 || ps_type > 2) return h->fail(CLB_EINVAL, "powerSpectrumType " + std::to_string(ps_type) + " is not a valid powerSpectrumType.");
  if (ps_version < 1 || ps_version > 2)
    return h->fail(CLB_EINVAL, "clb_spectrum: PS_version 1 (bin mean |k|) and 2 (bin centre) are supported");
  if (!(dk > 0) || nbins < 1) return h->fail(CLB_EINVAL, "clb_spectrum: dk must be positive and nbins >= 1");
  if (!value_out) return h->fail(CLB_EINVAL, "clb_spectrum: null output");
  const int N = h->N;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_spectrum");
  const size_t spec_n = (size_t)N * N * 2 * (N / 2 + 1);
  if (!h->d_spec) {
    if ((e = cudaMalloc(&h->d_spec, spec_n * sizeof(double))) != cudaSuccess)
      return h->fail(CLB_ENOMEM, std::string("clb_spectrum: ") + cudaGetErrorString(e));
  }
  if (!h->plan_ok) {
    if (cufftPlan3d(&h->plan, N, N, N, CUFFT_D2Z) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, "clb_spectrum: cufftPlan3d failed");
    h->plan_ok = true;
    if (cufftSetStream(h->plan, h->stream) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, "clb_spectrum: cufftSetStream failed");
  }
  if (nbins > h->spec_nbins_cap) {
    if (h->d_spec_part) cudaFree(h->d_spec_part);
    if (h->d_spec_cnt) cudaFree(h->d_spec_cnt);
    if (h->d_spec_out) cudaFree(h->d_spec_out);
    if (h->d_spec_outc) cudaFree(h->d_spec_outc);
    h->d_spec_part = nullptr;
    h->d_spec_cnt = nullptr;
    h->d_spec_out = nullptr;
    h->d_spec_outc = nullptr;
    bool ok = cudaMalloc(&h->d_spec_part, (size_t)kSpecBlocks * nbins * 2 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->d_spec_cnt, (size_t)kSpecBlocks * nbins * sizeof(unsigned long long)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->d_spec_out, (size_t)nbins * 2 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->d_spec_outc, (size_t)nbins * sizeof(unsigned long long)) == cudaSuccess;
    if (!ok) {
      h->spec_nbins_cap = 0;
      return h->fail(CLB_ENOMEM, "clb_spectrum: scratch allocation failed");
    }
    h->spec_nbins_cap = nbins;
  }
  if (plain) {
    CLB_LAUNCH(h, K_SPECTRUM, k_spec_gather_plain<<<kElemBlocks, 256, 0, h->stream>>>(plain, h->d_spec, N));
  } else {
    void *src = which == 0 ? h->fld[h->cf] : h->pi[h->cp];
    const size_t comp_off = (size_t)comp * (size_t)h->pd.comp;
    double ref = 0.0;
    if (h->fp32) {
      DevState cur;
      if ((e = cudaMemcpy(&cur, h->d_st, sizeof(cur), cudaMemcpyDeviceToHost)) != cudaSuccess) return h->cuda_fail(e, "clb_spectrum");
      ref = which == 0 ? cur.ref_phi[h->rs][comp] : cur.ref_pi[h->rs][comp];
      CLB_LAUNCH(h, K_SPECTRUM, k_spec_gather<float><<<kElemBlocks, 256, 0, h->stream>>>(static_cast<const float *>(src) + comp_off, h->d_spec, h->pd, ref));
    } else {
      CLB_LAUNCH(h, K_SPECTRUM, k_spec_gather<double><<<kElemBlocks, 256, 0, h->stream>>>(static_cast<const double *>(src) + comp_off, h->d_spec, h->pd, ref));
    }
  }
  if (cufftExecD2Z(h->plan, h->d_spec, reinterpret_cast<cufftDoubleComplex *>(h->d_spec)) != CUFFT_SUCCESS)
    return h->fail(CLB_ECUDA, "clb_spectrum: cufftExecD2Z failed");
  const size_t smem = (size_t)nbins * (2 * sizeof(double) + sizeof(unsigned long long));
  static size_t smem_attr = 0;
  if (smem > 48 * 1024 && smem > smem_attr) {
    if ((e = cudaFuncSetAttribute(k_spec_bin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
      return h->fail(CLB_EINVAL, "clb_spectrum: too many bins for shared memory");
    smem_attr = smem;
  }
  CLB_LAUNCH(h, K_SPECTRUM,
             k_spec_bin<<<kSpecBlocks, 256, smem, h->stream>>>(reinterpret_cast<const double2 *>(h->d_spec), N, dk, nbins,
                                                                 fold, h->d_spec_part, h->d_spec_cnt));
  CLB_LAUNCH(h, K_SPECTRUM,
             k_spec_sum<<<(nbins + 255) / 256, 256, 0, h->stream>>>(h->d_spec_part, h->d_spec_cnt, kSpecBlocks, nbins,
                                                                    h->d_spec_out, h->d_spec_out + nbins, h->d_spec_outc));
  sums.assign(2 * (size_t)nbins, 0.0);
  cnt.assign(nbins, 0ull);
  gauge_comp_out = gauge_comp;
  e = cudaMemcpyAsync(sums.data(), h->d_spec_out, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(cnt.data(), h->d_spec_outc, cnt.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_spectrum");
  collect_profile(h);
  double aI = 1.0;
  if (gauge_model) {
    clb_scalefactor sf;
    const int r = h->u1 ? u1_get_state(h, nullptr, nullptr, &sf) : su2_get_state(h, nullptr, nullptr, &sf);
    if (r != CLB_OK) return r;
    aI = sf.aI;
  } else {
    DevState s;
    if ((e = cudaMemcpy(&s, h->d_st, sizeof(s), cudaMemcpyDeviceToHost)) != cudaSuccess) return h->cuda_fail(e, "clb_spectrum");
    aI = s.aI;
  }
  const double kIR = 2 * 3.14159265358979323846 / (N * h->cfg.dx);
  // momenta: a^{2 alpha - 6} for matter (scalarsingletmeasurer.h:80), a^{2 alpha - 2} for gauge
  // components (u1measurer.h:102-103)
  const double mom_factor = which == 1 ? std::pow(aI, 2 * h->md.alpha - (gauge_comp ? 2 : 6)) : 1.0;
  for (int b = 0; b < nbins; ++b) {
    const unsigned long long c = cnt[b];
    double ntil;
    value_out[b] = mom_factor * spec_value(h, ps_type, ps_version, dk, b, c, sums[nbins + b], sums[b], &ntil);
    if (k_out) k_out[b] = ntil * kIR;
    if (count_out) count_out[b] = (int64_t)c;
  }
  return CLB_OK;
}

} // namespace

extern "C" {

int clb_spectrum(clb_handle *h, int32_t which, int32_t comp, int32_t ps_type, int32_t ps_version, double dk,
                 int32_t nbins, int32_t fold, double *k_out, double *value_out, int64_t *count_out)
{
  if (!h) return CLB_EINVAL;
  std::vector<double> sums;
  std::vector<unsigned long long> cnt;
  bool gauge_comp = false;
  return spectrum_impl(h, which, comp, ps_type, ps_version, dk, nbins, fold, k_out, value_out, count_out, sums, cnt,
                       gauge_comp);
}

// clb_forward with the observable O = sum_b w_b P_b, P the clb_spectrum of one component at the
// end state; the following clb_backward returns dO.
int clb_forward_spectrum(clb_handle *h, int64_t nsteps, int32_t checkpoint_every, int32_t which, int32_t comp,
                         int32_t ps_type, int32_t ps_version, double dk, int32_t nbins, int32_t fold,
                         const double *bin_weights, double *observable)
{
  if (!h) return CLB_EINVAL;
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_forward_spectrum: call clb_initialize first");
  if (!h->u1) return h->fail(CLB_EUNSUPPORTED, "clb_forward_spectrum: the adjoint pair covers lphi4U1");
  if (!bin_weights || nbins < 1) return h->fail(CLB_EINVAL, "clb_forward_spectrum: one weight per bin");
  int r = u1_forward(h, nsteps, checkpoint_every, nullptr, 0, nullptr);
  if (r != CLB_OK) return r;
  // the end state's spectrum: its bin sums and counts, and the component's transform in d_spec
  std::vector<double> sums, vals((size_t)nbins);
  std::vector<unsigned long long> cnt;
  bool gauge = false;
  r = spectrum_impl(h, which, comp, ps_type, ps_version, dk, nbins, fold, nullptr, vals.data(), nullptr, sums, cnt, gauge);
  if (r != CLB_OK) return r;
  clb_scalefactor sf;
  if ((r = u1_get_state(h, nullptr, nullptr, &sf)) != CLB_OK) return r;
  const double ex = 2 * h->md.alpha - (gauge ? 2 : 6);
  const double m = which == 1 ? std::pow(sf.aI, ex) : 1.0;
  double O = 0;
  std::vector<double> g((size_t)nbins);
  for (int b = 0; b < nbins; ++b) {
    O += bin_weights[b] * vals[(size_t)b];
    double ntil;
    g[(size_t)b] = bin_weights[b] * m * spec_value(h, ps_type, ps_version, dk, b, cnt[(size_t)b], sums[(size_t)nbins + b], 1.0, &ntil);
  }
  const double abar = which == 1 ? ex * O / sf.aI : 0.0; // dO/da through the momentum spectra's a-factor
  // dO/d(component) = 2 C2R(g f_k)
  const int N = h->N;
  const size_t spec_n = (size_t)N * N * 2 * (N / 2 + 1);
  cudaError_t e = cudaSuccess;
  if (!h->d_spec2 && (e = cudaMalloc(&h->d_spec2, spec_n * sizeof(double))) != cudaSuccess)
    return h->fail(CLB_ENOMEM, std::string("clb_forward_spectrum: ") + cudaGetErrorString(e));
  if (!h->plan_inv_ok) {
    if (cufftPlan3d(&h->plan_inv, N, N, N, CUFFT_Z2D) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, "clb_forward_spectrum: cufftPlan3d failed");
    h->plan_inv_ok = true;
    if (cufftSetStream(h->plan_inv, h->stream) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, "clb_forward_spectrum: cufftSetStream failed");
  }
  double *d_g = h->d_spec_out; // nbins x 2 doubles of scratch (the bin sums are on the host by now)
  if ((e = cudaMemcpyAsync(d_g, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
    return h->cuda_fail(e, "clb_forward_spectrum");
  CLB_LAUNCH(h, K_SPECTRUM, k_spec_weight<<<kSpecBlocks, 256, 0, h->stream>>>(reinterpret_cast<double2 *>(h->d_spec), N, dk,
                                                                             nbins, fold, d_g));
  if (cufftExecZ2D(h->plan_inv, reinterpret_cast<cufftDoubleComplex *>(h->d_spec), h->d_spec) != CUFFT_SUCCESS)
    return h->fail(CLB_ECUDA, "clb_forward_spectrum: cufftExecZ2D failed");
  CLB_LAUNCH(h, K_SPECTRUM, k_spec_extract<<<kElemBlocks, 256, 0, h->stream>>>(h->d_spec, h->d_spec2, N, 2.0));
  if ((e = cudaGetLastError()) != cudaSuccess) return h->cuda_fail(e, "clb_forward_spectrum");
  if ((r = u1_set_spectrum_seed(h, which, comp, h->d_spec2, O, abar)) != CLB_OK) return r;
  if (observable) *observable = O;
  return CLB_OK;
}

// clb_spectrum of a component and its derivative along the tangent-linear form's direction.
int clb_tangent_spectrum(clb_handle *h, int32_t which, int32_t comp, int32_t ps_type, int32_t ps_version, double dk,
                         int32_t nbins, int32_t fold, double *k_out, double *value_out, double *d_value_out,
                         int64_t *count_out)
{
  if (!h) return CLB_EINVAL;
  if (!h->su2) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_spectrum: the tangent-linear form covers lphi4SU2U1");
  if (!d_value_out) return h->fail(CLB_EINVAL, "clb_tangent_spectrum: null output");
  bool f32 = false;
  double aI = 1, daI = 0;
  const void *tsrc = nullptr;
  if (which == 0 || which == 1) tsrc = su2_tangent_component(h, which, comp, &f32, &aI, &daI);
  if (!tsrc && (which == 0 || which == 1) && comp >= 0 && comp < (which == 0 ? 22 : 19))
    return h->fail(CLB_ESTATE, "clb_tangent_spectrum: call clb_tangent_begin first");
  std::vector<double> sums;
  std::vector<unsigned long long> cnt;
  bool gauge_comp = false;
  int r = spectrum_impl(h, which, comp, ps_type, ps_version, dk, nbins, fold, k_out, value_out, count_out, sums, cnt,
                        gauge_comp);
  if (r != CLB_OK) return r;
  // the component's transform is in d_spec; transform its tangent into d_spec2
  const int N = h->N;
  const size_t spec_n = (size_t)N * N * 2 * (N / 2 + 1);
  cudaError_t e = cudaSuccess;
  if (!h->d_spec2 && (e = cudaMalloc(&h->d_spec2, spec_n * sizeof(double))) != cudaSuccess)
    return h->fail(CLB_ENOMEM, std::string("clb_tangent_spectrum: ") + cudaGetErrorString(e));
  if (f32)
    CLB_LAUNCH(h, K_SPECTRUM, k_spec_gather_raw<float><<<kElemBlocks, 256, 0, h->stream>>>(static_cast<const float *>(tsrc), h->d_spec2, N));
  else
    CLB_LAUNCH(h, K_SPECTRUM, k_spec_gather_raw<double><<<kElemBlocks, 256, 0, h->stream>>>(static_cast<const double *>(tsrc), h->d_spec2, N));
  if (cufftExecD2Z(h->plan, h->d_spec2, reinterpret_cast<cufftDoubleComplex *>(h->d_spec2)) != CUFFT_SUCCESS)
    return h->fail(CLB_ECUDA, "clb_tangent_spectrum: cufftExecD2Z failed");
  const size_t smem = (size_t)nbins * sizeof(double);
  if (smem > 48 * 1024 && (e = cudaFuncSetAttribute(k_spec_bin_cross, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
    return h->fail(CLB_EINVAL, "clb_tangent_spectrum: too many bins for shared memory");
  CLB_LAUNCH(h, K_SPECTRUM,
             k_spec_bin_cross<<<kSpecBlocks, 256, smem, h->stream>>>(reinterpret_cast<const double2 *>(h->d_spec),
                                                                     reinterpret_cast<const double2 *>(h->d_spec2), N,
                                                                     dk, nbins, fold, h->d_spec_part, h->d_spec_cnt));
  CLB_LAUNCH(h, K_SPECTRUM,
             k_spec_sum<<<(nbins + 255) / 256, 256, 0, h->stream>>>(h->d_spec_part, h->d_spec_cnt, kSpecBlocks, nbins,
                                                                    h->d_spec_out, h->d_spec_out + nbins, h->d_spec_outc));
  std::vector<double> dsum((size_t)nbins);
  e = cudaMemcpyAsync(dsum.data(), h->d_spec_out, dsum.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_tangent_spectrum");
  collect_profile(h);
  // value = m(a) S(sum): d value = m dS(dsum) + m' da S(sum), m = a^{2 alpha - 6} (matter momenta),
  // a^{2 alpha - 2} (gauge momenta), 1 (fields)
  const double ex = 2 * h->md.alpha - (gauge_comp ? 2 : 6);
  const double m = which == 1 ? std::pow(aI, ex) : 1.0;
  const double dm = which == 1 ? ex * std::pow(aI, ex - 1) * daI : 0.0;
  for (int b = 0; b < nbins; ++b) {
    double ntil;
    const double v = spec_value(h, ps_type, ps_version, dk, b, cnt[b], sums[nbins + b], sums[b], &ntil);
    const double dv = spec_value(h, ps_type, ps_version, dk, b, cnt[b], sums[nbins + b], dsum[b], &ntil);
    d_value_out[b] = m * dv + dm * v;
  }
  return CLB_OK;
}

} // extern "C"
