// clb_gws.cu - the gravitational-wave sector: its C ABI, the scalar singlets' source, and the
// energy spectrum.  The kick and drift kernels are in clb_gws.cuh; the gauge models' sources are in
// clb_u1.cu (lphi4U1) and clb_su2.cu (lphi4SU2U1).
//
// The GW field is the traceless symmetric u_ij stored as five components (u_11, u_12, u_13, u_22,
// u_23; u_33 = -u_11 - u_22, the storage gwsprojector.h reads), zero at the start
// (GWsInitializer, gwsinitializer.h).  With the reference's default (doLFforGWs, runparameters.h:121)
// it advances as a leapfrog staggered over the matter evolver (Evolver::evolve, evolver.h:102-124):
//   before each matter step  pi_u += (w dt) K(u, source; a_I),  w = 1/2 after a sync, else 1
//   after it                 u += pow(a_SI, alpha - 3) (dt pi_u)
// and Evolver::sync (evolver.h:132-138) kicks by dt/2 to integer time before a measurement.  The
// kernel (GWsKernels::get, gwskernels.h:27-33) is
//   K = a^(1+alpha) lapl(u) + a^(1+alpha) 2 Pi,
// with lapl the seven-point Laplacian of each component (gaugederivatives.h:42-46) and Pi the
// anisotropic tensor of PITensor.h: the scalar singlets' sum_a forwDiff_i phi_a forwDiff_j phi_a,
// the complex scalars' 2 Re[D_i phi conj(D_j phi)] and the U(1) electric and magnetic terms.  The
// five stored components take its traceless part (Pi_11 - tr/3, Pi_12, Pi_13, Pi_22 - tr/3,
// Pi_23; TempLat's ConstructSymTraceless is not vendored: a stated choice, and the TT projection
// of the measurement removes the trace either way).  The SU(2) doublet and the SU(2) gauge field
// source no GWs in PITensor.h, and none here.  FP64 pins every rounding in the order above; the
// oracle restates it.
//
// The energy spectrum (PowerSpectrumMeasurer::powerSpectrumGW, powerspectrum.h:51-71;
// GWsMeasurer, gwsmeasurer.h) transforms the five momentum components, projects each mode with
// the TT projector of GWProjectorType1/2/3 (gwsprojector.h), bins like clb_spectrum and scales by
// (fStar/MPl)^2 / (4 a^6 rho).  The zero mode, where the lattice momentum vanishes and the
// projector is undefined, contributes nothing.
#include "../../include/clb200.h"
#include "clb_gws.cuh"
#include "clb_handle.cuh"
#include "clb_internal.cuh"
#include "clb_scalar.cuh"
#include "clb_spectrum.cuh"
#include "clb_sweep.cuh"
#include "clb_vv.h"

#include <cmath>
#include <string>
#include <vector>

namespace {

constexpr int kGWSpecBlocks = 148 * 2;

// The scalar-singlet source of PITensor.h: Pi_ij = sum_a forwDiff_i phi_a forwDiff_j phi_a, from the
// padded field layout.
template <class R, int NS> struct ScalarGWSource {
  const R *fld;
  Pad pd;
  R dx;
  __device__ __forceinline__ void operator()(size_t, int x, int y, int z, int xp, int yp, int zp, R (&P)[6]) const
  {
    using A = Ar<R>;
#pragma unroll
    for (int f = 0; f < NS; ++f) {
      const R *F = fld + (size_t)f * pd.comp;
      const R c = F[pd.at(x, y, z)];
      const R g0 = A::sub(F[pd.at(xp, y, z)], c) / dx, g1 = A::sub(F[pd.at(x, yp, z)], c) / dx,
              g2 = A::sub(F[pd.at(x, y, zp)], c) / dx;
      const R t[6] = {A::mul(g0, g0), A::mul(g0, g1), A::mul(g0, g2), A::mul(g1, g1), A::mul(g1, g2), A::mul(g2, g2)};
#pragma unroll
      for (int k = 0; k < 6; ++k) P[k] = f == 0 ? t[k] : A::add(P[k], t[k]);
    }
  }
};

// The TT-projected power of one mode (GWProjectorType1/2/3::eval, gwsprojector.h).
struct Cx {
  double re, im;
};
__device__ __forceinline__ Cx cx_mul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cx cx_add(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx cx_sub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx cx_conj(Cx a) { return {a.re, -a.im}; }

__device__ void gw_pu(const Cx (&P)[6], const Cx (&u)[5], Cx (&Pu)[9])
{
  const Cx t = cx_add(u[0], u[3]);
  Pu[0] = cx_add(cx_add(cx_mul(P[0], u[0]), cx_mul(P[1], u[1])), cx_mul(P[2], u[2]));
  Pu[1] = cx_add(cx_add(cx_mul(P[0], u[1]), cx_mul(P[1], u[3])), cx_mul(P[2], u[4]));
  Pu[2] = cx_sub(cx_add(cx_mul(P[0], u[2]), cx_mul(P[1], u[4])), cx_mul(P[2], t));
  Pu[3] = cx_add(cx_add(cx_mul(cx_conj(P[1]), u[0]), cx_mul(P[3], u[1])), cx_mul(P[4], u[2]));
  Pu[4] = cx_add(cx_add(cx_mul(cx_conj(P[1]), u[1]), cx_mul(P[3], u[3])), cx_mul(P[4], u[4]));
  Pu[5] = cx_sub(cx_add(cx_mul(cx_conj(P[1]), u[2]), cx_mul(P[3], u[4])), cx_mul(P[4], t));
  Pu[6] = cx_add(cx_add(cx_mul(cx_conj(P[2]), u[0]), cx_mul(cx_conj(P[4]), u[1])), cx_mul(P[5], u[2]));
  Pu[7] = cx_add(cx_add(cx_mul(cx_conj(P[2]), u[1]), cx_mul(cx_conj(P[4]), u[3])), cx_mul(P[5], u[4]));
  Pu[8] = cx_sub(cx_add(cx_mul(cx_conj(P[2]), u[2]), cx_mul(cx_conj(P[4]), u[4])), cx_mul(P[5], t));
}

__device__ double gw_mode(const Cx (&u)[5], long long nx, long long ny, long long nz, int N, int prj)
{
  const double kir = 2.0 * 3.14159265358979323846 / N;
  const long long n[3] = {nx, ny, nz};
  Cx kL[3];
  for (int i = 0; i < 3; ++i) {
    const double a = kir * (double)n[i];
    kL[i] = prj == 1 ? Cx{sin(a), 0.0} : Cx{sin(a), (prj == 2 ? -1.0 : 1.0) * (1.0 - cos(a))};
  }
  const double kL2 = (kL[0].re * kL[0].re + kL[0].im * kL[0].im) + (kL[1].re * kL[1].re + kL[1].im * kL[1].im) +
                     (kL[2].re * kL[2].re + kL[2].im * kL[2].im);
  if (kL2 == 0.0) return 0.0;
  auto pp = [&](int i, int j, bool diag) {
    const Cx q = cx_mul(cx_conj(kL[i]), kL[j]);
    return diag ? Cx{1.0 - q.re / kL2, -q.im / kL2} : Cx{-q.re / kL2, -q.im / kL2};
  };
  const Cx P[6] = {pp(0, 0, true), pp(0, 1, false), pp(0, 2, false), pp(1, 1, true), pp(1, 2, false), pp(2, 2, true)};
  Cx uc[5];
  for (int c = 0; c < 5; ++c) uc[c] = cx_conj(u[c]);
  Cx Pu[9], Pus[9];
  gw_pu(P, u, Pu);
  gw_pu(P, uc, Pus);
  Cx Tr1 = cx_mul(Pu[0], Pus[0]);
  const int a[8] = {1, 2, 3, 4, 5, 6, 7, 8}, b[8] = {3, 6, 1, 4, 7, 2, 5, 8};
  for (int k = 0; k < 8; ++k) Tr1 = cx_add(Tr1, cx_mul(Pu[a[k]], Pus[b[k]]));
  const Cx Tr2 = cx_add(cx_add(Pu[0], Pu[4]), Pu[8]), Tr2s = cx_add(cx_add(Pus[0], Pus[4]), Pus[8]);
  const Cx d = cx_mul(Tr2, Tr2s);
  const Cx r = {Tr1.re - 0.5 * d.re, Tr1.im - 0.5 * d.im};
  return sqrt(r.re * r.re + r.im * r.im);
}

// k_spec_bin's binning of the projected power over the five transforms (nzh = N/2 + 1 per row).
__global__ void __launch_bounds__(256)
    k_gw_bin(const double2 *__restrict__ fk, size_t comp_stride, int N, double dk, int nbins, int fold, int prj,
             double *__restrict__ part_val, unsigned long long *__restrict__ part_cnt)
{
  extern __shared__ unsigned char smem_raw[];
  double *h_val = reinterpret_cast<double *>(smem_raw);
  double *h_n = h_val + nbins;
  unsigned long long *h_cnt = reinterpret_cast<unsigned long long *>(h_n + nbins);
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
    h_val[b] = 0.0;
    h_n[b] = 0.0;
    h_cnt[b] = 0ull;
  }
  __syncthreads();
  const int nzh = N / 2 + 1;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int kx = (int)(r / N), ky = (int)(r % N);
    // the Nyquist index stands for n = +N/2 (at the corner mode the type-1 momenta are three
    // rounding-sized sin(pi) values whose signs set the projector)
    const long long nx = kx <= N / 2 ? kx : kx - N;
    const long long ny = ky <= N / 2 ? ky : ky - N;
    for (int kz = threadIdx.x; kz < nzh; kz += blockDim.x) {
      const long long n2 = nx * nx + ny * ny + (long long)kz * kz;
      const double nn = sqrt((double)n2);
      int b = (int)floor(nn / dk);
      if (b >= nbins) {
        if (!fold) continue;
        b = nbins - 1;
      }
      Cx u[5];
      for (int c = 0; c < 5; ++c) {
        const double2 v = fk[c * comp_stride + r * nzh + kz];
        u[c] = {v.x, v.y};
      }
      const int w = (kz == 0 || (2 * kz == N)) ? 1 : 2;
      atomicAdd(&h_val[b], w * gw_mode(u, nx, ny, kz, N, prj));
      atomicAdd(&h_n[b], w * nn);
      atomicAdd(&h_cnt[b], (unsigned long long)w);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
    part_val[((size_t)blockIdx.x * nbins + b) * 2 + 0] = h_val[b];
    part_val[((size_t)blockIdx.x * nbins + b) * 2 + 1] = h_n[b];
    part_cnt[(size_t)blockIdx.x * nbins + b] = h_cnt[b];
  }
}

// Host-order (5 x N^3 doubles) <-> storage-type arrays.
template <class S, class D> __global__ void __launch_bounds__(256) k_gw_copy(const S *src, D *dst, size_t n)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (D)src[i];
}

bool gw_ok(const clb_handle *h) { return h->gw != nullptr; }

} // namespace

namespace clb {

// The gauge models' GW kick and drift (clb_u1.cu, clb_su2.cu).
void u1_gw_kick(clb_handle *h, double w);
void u1_gw_drift(clb_handle *h);
void su2_gw_kick(clb_handle *h, double w);
void su2_gw_drift(clb_handle *h);
bool su2_tangent_active(const clb_handle *h);

// Runs one GW kick (weight w of dt) at the handle's current fields and a_I.
__attribute__((visibility("hidden"))) void gw_kick(clb_handle *h, double w)
{
  GWSector *g = h->gw;
  g->synced = false;
  if (h->u1) return u1_gw_kick(h, w);
  if (h->su2) return su2_gw_kick(h, w);
  const double inv_dx2 = 1.0 / (h->cfg.dx * h->cfg.dx);
  const double hd = w * h->cfg.dt;
#define CLB_GWK(R, NS)                                                                                                 \
  CLB_LAUNCH(h, K_GW, (k_gw_kick<R, ScalarGWSource<R, NS>><<<kGWBlocks, 256, 0, h->stream>>>(                        \
                          static_cast<const R *>(g->u), static_cast<R *>(g->pi), h->N, inv_dx2, hd, &h->d_st->kick_A, \
                          ScalarGWSource<R, NS>{static_cast<const R *>(h->fld[h->cf]), h->pd, (R)h->cfg.dx})))
  if (h->fp32) {
    if (h->NS == 1) CLB_GWK(float, 1);
    else CLB_GWK(float, 2);
  } else {
    if (h->NS == 1) CLB_GWK(double, 1);
    else CLB_GWK(double, 2);
  }
#undef CLB_GWK
}

// Runs one GW drift with the a_SI of the matter step just taken.
__attribute__((visibility("hidden"))) void gw_drift(clb_handle *h)
{
  if (h->u1) return u1_gw_drift(h);
  if (h->su2) return su2_gw_drift(h);
  GWSector *g = h->gw;
  const size_t n = 5 * h->n3;
  const bool pv = is_pv(h->cfg.evolver);
  if (h->fp32)
    CLB_LAUNCH(h, K_GW, launch_gw_drift<float>(static_cast<float *>(g->u), static_cast<const float *>(g->pi), n,
                                               h->cfg.dt, &h->d_st->drift_p, &h->d_st->aSI, h->md.alpha, pv,
                                               h->stream));
  else
    CLB_LAUNCH(h, K_GW, launch_gw_drift<double>(static_cast<double *>(g->u), static_cast<const double *>(g->pi), n,
                                                h->cfg.dt, &h->d_st->drift_p, &h->d_st->aSI, h->md.alpha, pv,
                                                h->stream));
}

// The GW kick before a matter step (evolver.h:104-107): half a step after a sync, else a whole one.
__attribute__((visibility("hidden"))) void gw_kick_step(clb_handle *h) { gw_kick(h, h->gw->synced ? 0.5 : 1.0); }

// Evolver::sync (evolver.h:132-138): the half kick to integer time, if the momenta are unsynced.
__attribute__((visibility("hidden"))) void gw_sync(clb_handle *h)
{
  if (!h->gw->synced) gw_kick(h, 0.5);
  h->gw->synced = true;
}

__attribute__((visibility("hidden"))) void gw_set_synced(clb_handle *h, bool s) { h->gw->synced = s; }

__attribute__((visibility("hidden"))) void gw_destroy(clb_handle *h)
{
  if (!h->gw) return;
  if (h->gw->u) cudaFree(h->gw->u);
  if (h->gw->pi) cudaFree(h->gw->pi);
  if (h->gw->d_fk) cudaFree(h->gw->d_fk);
  delete h->gw;
  h->gw = nullptr;
}

} // namespace clb

extern "C" {

int clb_gws_enable(clb_handle *h)
{
  if (!h) return CLB_EINVAL;
  if (h->gw) return CLB_OK;
  const bool gauge = h->u1 || h->su2;
  if (!gauge && h->cfg.path != CLB_PATH_FUSED)
    return h->fail(CLB_EUNSUPPORTED, "clb_gws_enable: the scalar singlets' GWs run on the fused path");
  if (h->su2 && su2_tangent_active(h))
    return h->fail(CLB_EUNSUPPORTED, "clb_gws_enable: not with the tangent-linear form running");
  auto *g = new GWSector();
  g->fp32 = gauge ? h->cfg.precision == CLB_PREC_FP32_SPLIT : h->fp32;
  const size_t bytes = 5 * h->n3 * (g->fp32 ? sizeof(float) : sizeof(double));
  cudaError_t e = cudaMalloc(&g->u, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&g->pi, bytes);
  if (e == cudaSuccess) e = cudaMemset(g->u, 0, bytes);
  if (e == cudaSuccess) e = cudaMemset(g->pi, 0, bytes);
  h->gw = g;
  if (e != cudaSuccess) {
    gw_destroy(h);
    return h->fail(CLB_ENOMEM, std::string("clb_gws_enable: ") + cudaGetErrorString(e));
  }
  return CLB_OK;
}

int clb_gws_set_state(clb_handle *h, const double *u, const double *pi)
{
  if (!h) return CLB_EINVAL;
  if (!gw_ok(h)) return h->fail(CLB_ESTATE, "clb_gws_set_state: call clb_gws_enable first");
  const size_t n = 5 * h->n3;
  double *tmp = nullptr;
  cudaError_t e = cudaMalloc(&tmp, n * sizeof(double));
  for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
    const double *src = k == 0 ? u : pi;
    void *dst = k == 0 ? h->gw->u : h->gw->pi;
    if (!src) continue;
    e = cudaMemcpyAsync(tmp, src, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) break;
    if (h->gw->fp32)
      k_gw_copy<double, float><<<kGWBlocks, 256, 0, h->stream>>>(tmp, static_cast<float *>(dst), n);
    else
      e = cudaMemcpyAsync(dst, tmp, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  }
  if (tmp) cudaFree(tmp);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_gws_set_state");
  return CLB_OK;
}

int clb_gws_get_state(clb_handle *h, double *u, double *pi)
{
  if (!h) return CLB_EINVAL;
  if (!gw_ok(h)) return h->fail(CLB_ESTATE, "clb_gws_get_state: call clb_gws_enable first");
  const size_t n = 5 * h->n3;
  double *tmp = nullptr;
  cudaError_t e = cudaMalloc(&tmp, n * sizeof(double));
  for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
    double *dst = k == 0 ? u : pi;
    const void *src = k == 0 ? h->gw->u : h->gw->pi;
    if (!dst) continue;
    if (h->gw->fp32)
      k_gw_copy<float, double><<<kGWBlocks, 256, 0, h->stream>>>(static_cast<const float *>(src), tmp, n);
    else
      e = cudaMemcpyAsync(tmp, src, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  }
  if (tmp) cudaFree(tmp);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_gws_get_state");
  return CLB_OK;
}

int clb_gw_spectrum(clb_handle *h, int32_t prj_type, int32_t ps_type, int32_t ps_version, double dk, int32_t nbins,
                    int32_t fold, double *k_out, double *value_out, int64_t *count_out, double *rho_gw_over_rho)
{
  if (!h) return CLB_EINVAL;
  if (!gw_ok(h)) return h->fail(CLB_ESTATE, "clb_gw_spectrum: call clb_gws_enable first");
  if (!h->initialized) return h->fail(CLB_ESTATE, "clb_gw_spectrum: call clb_initialize first");
  if (prj_type < 1 || prj_type > 3) return h->fail(CLB_EINVAL, "clb_gw_spectrum: GWprojectorType is 1, 2 or 3");
  if (ps_type < 1 || ps_type > 2 || ps_version < 1 || ps_version > 2 || !(dk > 0) || nbins < 1 || !value_out)
    return h->fail(CLB_EINVAL, "clb_gw_spectrum: PS_type 1 or 2, PS_version 1 or 2, dk > 0, nbins >= 1, an output");
  // Energies::rho at the current state (refreshes the cached averages, as the reference's does)
  clb_measurement m{};
  int r = clb_measure(h, 1.0, &m);
  if (r != CLB_OK) return r;
  const double rho = m.energies[m.n_energies - 1];
  const int N = h->N;
  const size_t nzh = (size_t)(N / 2 + 1);
  const size_t comp_n = (size_t)N * N * 2 * nzh; // doubles per in-place D2Z buffer
  cudaError_t e = cudaSuccess;
  if (!h->gw->d_fk && (e = cudaMalloc(&h->gw->d_fk, 5 * comp_n * sizeof(double))) != cudaSuccess)
    return h->fail(CLB_ENOMEM, std::string("clb_gw_spectrum: ") + cudaGetErrorString(e));
  if (!h->plan_ok) {
    if (cufftPlan3d(&h->plan, N, N, N, CUFFT_D2Z) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, "clb_gw_spectrum: cufftPlan3d failed");
    h->plan_ok = true;
    if (cufftSetStream(h->plan, h->stream) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, "clb_gw_spectrum: cufftSetStream failed");
  }
  for (int c = 0; c < 5; ++c) {
    double *dst = h->gw->d_fk + (size_t)c * comp_n;
    if (h->gw->fp32)
      CLB_LAUNCH(h, K_SPECTRUM, k_spec_gather_raw<float><<<kGWBlocks, 256, 0, h->stream>>>(
                                    static_cast<const float *>(h->gw->pi) + (size_t)c * h->n3, dst, N));
    else
      CLB_LAUNCH(h, K_SPECTRUM, k_spec_gather_raw<double><<<kGWBlocks, 256, 0, h->stream>>>(
                                    static_cast<const double *>(h->gw->pi) + (size_t)c * h->n3, dst, N));
    if (cufftExecD2Z(h->plan, dst, reinterpret_cast<cufftDoubleComplex *>(dst)) != CUFFT_SUCCESS)
      return h->fail(CLB_ECUDA, "clb_gw_spectrum: cufftExecD2Z failed");
  }
  double *part_val = nullptr, *out = nullptr;
  unsigned long long *part_cnt = nullptr, *outc = nullptr;
  e = cudaMalloc(&part_val, (size_t)kGWSpecBlocks * nbins * 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&part_cnt, (size_t)kGWSpecBlocks * nbins * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&out, (size_t)nbins * 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&outc, (size_t)nbins * sizeof(unsigned long long));
  std::vector<double> sums(2 * (size_t)nbins);
  std::vector<unsigned long long> cnt((size_t)nbins);
  const size_t smem = (size_t)nbins * (2 * sizeof(double) + sizeof(unsigned long long));
  if (e == cudaSuccess && smem > 48 * 1024)
    e = cudaFuncSetAttribute(k_gw_bin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    CLB_LAUNCH(h, K_SPECTRUM, k_gw_bin<<<kGWSpecBlocks, 256, smem, h->stream>>>(
                                  reinterpret_cast<const double2 *>(h->gw->d_fk), comp_n / 2, N, dk, nbins, fold,
                                  prj_type, part_val, part_cnt));
    CLB_LAUNCH(h, K_SPECTRUM, k_spec_sum<<<(nbins + 255) / 256, 256, 0, h->stream>>>(part_val, part_cnt, kGWSpecBlocks,
                                                                                   nbins, out, out + nbins, outc));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(sums.data(), out, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), outc, cnt.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  for (void *p : {(void *)part_val, (void *)part_cnt, (void *)out, (void *)outc})
    if (p) cudaFree(p);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_gw_spectrum");
  // the PS normalisation of clb_spectrum, then (fStar/MPl)^2 / (4 a^6 rho) (powerspectrum.h:58)
  const double pi = 3.14159265358979323846;
  const double dx = h->cfg.dx, kIR = 2 * pi / (N * dx);
  double N5 = 1;
  for (int i = 0; i < 5; ++i) N5 *= (double)N;
  const double fm = h->md.fStar / h->md.MPl;
  const double a6 = std::pow(m.aI, 6);
  const double fac = fm * fm / (4.0 * a6 * rho);
  double frac = 0;
  for (int b = 0; b < nbins; ++b) {
    const unsigned long long c = cnt[(size_t)b];
    const double ntil = (ps_version == 1 && c > 0) ? sums[(size_t)nbins + b] / (double)c : (b + 0.5) * dk;
    double v = 0;
    if (c > 0) {
      if (ps_type == 1) {
        v = kIR * ntil * dx / dk / N5 / 2.0 / pi * sums[(size_t)b];
      } else {
        const double t = kIR * ntil * dx / N;
        v = t * t * t / dk / 2.0 / (pi * pi) * (sums[(size_t)b] / (double)c);
      }
    }
    v *= fac;
    value_out[b] = v;
    if (k_out) k_out[b] = ntil * kIR;
    if (count_out) count_out[b] = (int64_t)c;
    if (c > 0 && ntil > 0) frac += v * dk / ntil; // sum of d(rho_GW/rho)/dln k over d ln k = dk / k
  }
  if (rho_gw_over_rho) *rho_gw_over_rho = frac;
  return CLB_OK;
}

} // extern "C"
