// clb_ic.cu - initial conditions generated on the device (clb_generate_state).
//
// The recipe is the reference's:
//   singlets          FluctuationsGenerator::getFluctuationsNorm / conjugateGaussianFluctuations
//                     (initializers/fluctuationsgenerator.h:39-71, 130-150);
//   complex scalar    U1Initializer::addFluctuationsCScalarFromPhases (initializers/u1initializer.h:157-230);
//   SU(2) doublet     SU2Initializer::addFluctuationsSU2DoubletFromPhases (initializers/su2initializer.h:115-186);
//   gauge momenta     the Gauss laws solved in momentum space with A = 0 and unit links
//                     (u1initializer.h:90-114, su2initializer.h:65-85);
//   homogeneous part  added afterwards (scalarsingletinitializer.h:41-77).
// Every component is one mode kernel over the half spectrum, one cuFFT Z2D and one copy-out; a Gauss
// solve is a charge-density kernel, one D2Z and three (solve kernel, Z2D, copy-out).  The finished
// state goes through the model's set_state from device memory.
//
// Random numbers: Philox4x64-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC11), key (seed, stream), counter (mode index, 0, 0, 0); one block of four 64-bit
// words per mode and stream, u = (word >> 11) 2^-53.  Streams: singlet i: 1 + i (left and right
// movers, Box-Muller from words 0-1 and 2-3); complex scalar: 16 (phases e00, e01, e10, Rayleigh
// amplitude 0), 17 (Rayleigh amplitude 1); doublet: 32 (Rayleigh amplitudes), 33 (left phases),
// 34 (right phase 0).  The kz = 0 and (even N) kz = N/2 planes are made Hermitian: a mode whose
// partner (-kx, -ky) has the smaller index takes the conjugate of the partner's values and a
// self-conjugate mode keeps its real part, so the field is the real transform of the drawn modes.

#include "clb_handle.cuh"

#include <cmath>
#include <string>
#include <vector>

namespace clb {
int u1_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf);
int su2_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf);
int scalar_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf,
                     const double *means);
} // namespace clb

namespace {

constexpr int kICBlocks = 148 * 8;
constexpr unsigned long long kPhiloxM0 = 0xD2E7470EE14C6C93ull, kPhiloxM1 = 0xCA5A826395121157ull;
constexpr unsigned long long kPhiloxW0 = 0x9E3779B97F4A7C15ull, kPhiloxW1 = 0xBB67AE8584CAA73Bull;
constexpr int kStreamSinglet = 1, kStreamComplex = 16, kStreamDoublet = 32;
constexpr double kSqrt2 = 1.4142135623730951;

struct Words {
  unsigned long long w[4];
};

__device__ __forceinline__ Words philox4x64(unsigned long long c0, unsigned long long k0, unsigned long long k1)
{
  unsigned long long c1 = 0, c2 = 0, c3 = 0;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned long long hi0 = __umul64hi(kPhiloxM0, c0), lo0 = kPhiloxM0 * c0;
    const unsigned long long hi1 = __umul64hi(kPhiloxM1, c2), lo1 = kPhiloxM1 * c2;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += kPhiloxW0;
    k1 += kPhiloxW1;
  }
  return {{c0, c1, c2, c3}};
}

__device__ __forceinline__ double unif(unsigned long long x) { return (double)(x >> 11) * 0x1.0p-53; }

struct Cx {
  double x, y;
};
__device__ __forceinline__ Cx operator+(Cx a, Cx b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ Cx operator-(Cx a, Cx b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ Cx operator*(Cx a, Cx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ Cx operator*(double s, Cx a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ Cx operator/(Cx a, double s) { return {a.x / s, a.y / s}; }
__device__ __forceinline__ Cx cconj(Cx a) { return {a.x, -a.y}; }
__device__ __forceinline__ Cx times_i(double s, Cx a) { return {-(s * a.y), s * a.x}; } // (i s) a

__device__ __forceinline__ Cx cis(double u)
{
  double s, c;
  sincospi(2.0 * u, &s, &c);
  return {c, s};
}
__device__ __forceinline__ double rayleigh(double u) { return sqrt(-2.0 * log1p(-u)); }

// One component's modes: kind 0 singlet comp, 1 complex-scalar component comp, 2 doublet component comp.
struct ModeArgs {
  int N;
  int kind, comp, which; // which: 0 field, 1 momentum
  unsigned long long seed;
  double kIR, kcut, A;   // A = amplitude (L / dx^2)^(3/2) / sqrt 2
  double m2c, m20;       // m^2 of this component and of component 0 of its multiplet
  double adot;
};

__device__ __forceinline__ double omega_of(double k, double m2) { return sqrt(k * k + (m2 > 0 ? m2 : 0.0)); }

// getFluctuationsNorm (fluctuationsgenerator.h:39-65): H(kcut - k) A / sqrt(2 omega_k)
__device__ __forceinline__ double norm_of(const ModeArgs &a, double k, double omega)
{
  return k <= a.kcut ? a.A / sqrt(2.0 * omega) : 0.0;
}

__device__ Cx mode_value(const ModeArgs &a, unsigned long long idx, double k)
{
  if (a.kind == 0) {
    const Words w = philox4x64(idx, a.seed, kStreamSinglet + a.comp);
    const double omega = omega_of(k, a.m2c), norm = norm_of(a, k, omega);
    const Cx fL = (norm * rayleigh(unif(w.w[0]))) * cis(unif(w.w[1]));
    const Cx fR = (norm * rayleigh(unif(w.w[2]))) * cis(unif(w.w[3]));
    const Cx phi = (fL + fR) / kSqrt2;
    if (a.which == 0) return phi;
    return times_i(omega, fL - fR) / kSqrt2 - a.adot * phi;
  }
  const double omega0 = omega_of(k, a.m20);
  const double norm = norm_of(a, k, omega_of(k, a.m2c));
  Cx ea, eb;
  double amp;
  if (a.kind == 1) {
    const Words w = philox4x64(idx, a.seed, kStreamComplex);
    const Cx e00 = cis(unif(w.w[0])), e01 = cis(unif(w.w[1]));
    if (a.comp == 0) {
      ea = e00;
      eb = e01;
      amp = norm * rayleigh(unif(w.w[3]));
    } else {
      const Cx e10 = cis(unif(w.w[2]));
      ea = e10;
      eb = e01 * e10 * cconj(e00);
      amp = norm * rayleigh(unif(philox4x64(idx, a.seed, kStreamComplex + 1).w[0]));
    }
  } else {
    const Words wl = philox4x64(idx, a.seed, kStreamDoublet + 1);
    const Cx l0 = cis(unif(wl.w[0]));
    const Cx r0 = cis(unif(philox4x64(idx, a.seed, kStreamDoublet + 2).w[0]));
    ea = cis(unif(wl.w[a.comp]));
    eb = r0 * ea * cconj(l0);
    amp = norm * rayleigh(unif(philox4x64(idx, a.seed, kStreamDoublet).w[a.comp]));
  }
  const Cx f = (amp * (ea + eb)) / 2.0;
  if (a.which == 0) return f;
  const Cx p = times_i(-(omega0 * amp), ea - eb) / 2.0;
  return a.kind == 1 ? p - a.adot * f : p - (a.adot * f) / kSqrt2;
}

// The half spectrum (N x N x (N/2 + 1)) of one component.
__global__ void __launch_bounds__(256) k_ic_modes(double2 *__restrict__ out, ModeArgs a)
{
  const int N = a.N, nzh = N / 2 + 1;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int kx = (int)(r / N), ky = (int)(r % N);
    const long long nx = kx <= N / 2 ? kx : kx - N;
    const long long ny = ky <= N / 2 ? ky : ky - N;
    const long long pr = (long long)((N - kx) % N) * N + (N - ky) % N;
    for (int kz = threadIdx.x; kz < nzh; kz += blockDim.x) {
      const long long n2 = nx * nx + ny * ny + (long long)kz * kz;
      const bool herm = kz == 0 || (N % 2 == 0 && 2 * kz == N);
      const unsigned long long idx = (unsigned long long)(r * nzh + kz), pidx = (unsigned long long)(pr * nzh + kz);
      Cx v{0.0, 0.0};
      if (n2 != 0) {
        const bool partner = herm && pidx < idx;
        v = mode_value(a, partner ? pidx : idx, sqrt((double)n2) * a.kIR);
        if (partner) v.y = -v.y;
        else if (herm && pidx == idx) v.y = 0.0;
      }
      out[r * nzh + kz] = make_double2(v.x, v.y);
    }
  }
}

// Real output of an in-place C2R transform (row pitch 2 (N/2 + 1)) -> scale x + add, N^3 plain.
__global__ void __launch_bounds__(256) k_ic_extract(const double *__restrict__ src, double *__restrict__ dst, int N,
                                                    double scale, double add)
{
  const long long pitch = 2LL * (N / 2 + 1);
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x)
    for (int z = threadIdx.x; z < N; z += blockDim.x) dst[r * N + z] = src[r * pitch + z] * scale + add;
}

// -dx^2 rho into the padded real layout of an in-place D2Z.  form 0: lphi4U1,
// rho = 2/dx r2 g (pi_0 phi_1 - pi_1 phi_0) (mattercurrents.h:27-48); form 1 + b: lphi4SU2U1 SU(2)
// component b, rho_b / dx with rho_b = r2/2 gS Re((i sigma_b Phi)^+ pi_Phi) (mattercurrents.h:86-98);
// form 4: lphi4SU2U1 U(1), rho = 2/dx r2 (gC (pi_1 phi_2 - pi_2 phi_1) + gD Im(pi_Phi^+ Phi)).
struct ChargeArgs {
  int N, form;
  size_t n3;
  double dx, r2, g0, g1;
};

__global__ void __launch_bounds__(256) k_ic_charge(const double *__restrict__ F, const double *__restrict__ P,
                                                   double *__restrict__ out, ChargeArgs a)
{
  const int N = a.N;
  const long long pitch = 2LL * (N / 2 + 1);
  const size_t n3 = a.n3;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x)
    for (int z = threadIdx.x; z < N; z += blockDim.x) {
      const size_t i = (size_t)r * N + z;
      double rho;
      if (a.form == 0) {
        rho = 2.0 / a.dx * a.r2 * a.g0 * (P[i] * F[n3 + i] - P[n3 + i] * F[i]);
      } else {
        const Cx u{F[3 * n3 + i], F[4 * n3 + i]}, v{F[5 * n3 + i], F[6 * n3 + i]};
        const Cx pu{P[3 * n3 + i], P[4 * n3 + i]}, pv{P[5 * n3 + i], P[6 * n3 + i]};
        if (a.form == 4) {
          const Cx s = cconj(pu) * u + cconj(pv) * v;
          rho = 2.0 / a.dx * a.r2 * (a.g0 * (P[n3 + i] * F[2 * n3 + i] - P[2 * n3 + i] * F[n3 + i]) + a.g1 * s.y);
        } else {
          // i sigma_b Phi for Phi = (u, v): b 0 (i v, i u), 1 (v, -u), 2 (i u, -i v)
          Cx ta, tc;
          if (a.form == 1) {
            ta = {-v.y, v.x};
            tc = {-u.y, u.x};
          } else if (a.form == 2) {
            ta = v;
            tc = {-u.x, -u.y};
          } else {
            ta = {-u.y, u.x};
            tc = {v.y, -v.x};
          }
          const Cx s = cconj(ta) * pu + cconj(tc) * pv;
          rho = a.r2 / 2 * (a.g0 * s.x) / a.dx;
        }
      }
      out[r * pitch + z] = -a.dx * a.dx * rho;
    }
}

// pi_dir = conj(q_dir) / sum_j |q_j|^2 j0, q_j = 1 - exp(-2 pi i n_j / N), zero mode 0.
__global__ void __launch_bounds__(256) k_ic_gauss(const double2 *__restrict__ j0, double2 *__restrict__ out, int N,
                                                  int dir)
{
  const int nzh = N / 2 + 1;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int kx = (int)(r / N), ky = (int)(r % N);
    const long long nx = kx <= N / 2 ? kx : kx - N;
    const long long ny = ky <= N / 2 ? ky : ky - N;
    for (int kz = threadIdx.x; kz < nzh; kz += blockDim.x) {
      const long long n[3] = {nx, ny, kz};
      Cx q[3];
      double k2 = 0;
      for (int j = 0; j < 3; ++j) {
        const Cx e = cis(-(double)n[j] / N);
        q[j] = {1.0 - e.x, -e.y};
        k2 += q[j].x * q[j].x + q[j].y * q[j].y;
      }
      const size_t m = (size_t)r * nzh + kz;
      Cx v{0.0, 0.0};
      if (nx != 0 || ny != 0 || kz != 0) v = (cconj(q[dir]) / k2) * Cx{j0[m].x, j0[m].y};
      out[m] = make_double2(v.x, v.y);
    }
  }
}

__global__ void __launch_bounds__(256) k_ic_fill(double *__restrict__ dst, size_t n, double v)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) dst[i] = v;
}

// Per-block sums of x (fixed order: strided per thread, then a tree over the block).
__global__ void __launch_bounds__(256) k_ic_sum(const double *__restrict__ x, size_t n, double *__restrict__ part)
{
  __shared__ double s[256];
  double acc = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) acc += x[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

struct Gen {
  clb_handle *h;
  const char *where = "clb_generate_state";
  int N;
  size_t n3, spec_n;
  ModeArgs base{};

  int ensure_fft()
  {
    cudaError_t e = cudaSuccess;
    if (!h->d_spec && (e = cudaMalloc(&h->d_spec, spec_n * sizeof(double))) != cudaSuccess)
      return h->fail(CLB_ENOMEM, std::string(where) + ": " + cudaGetErrorString(e));
    if (!h->d_spec2 && (e = cudaMalloc(&h->d_spec2, spec_n * sizeof(double))) != cudaSuccess)
      return h->fail(CLB_ENOMEM, std::string(where) + ": " + cudaGetErrorString(e));
    if (!h->plan_ok) {
      if (cufftPlan3d(&h->plan, N, N, N, CUFFT_D2Z) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, std::string(where) + ": cufftPlan3d failed");
      h->plan_ok = true;
      if (cufftSetStream(h->plan, h->stream) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, std::string(where) + ": cufftSetStream failed");
    }
    if (!h->plan_inv_ok) {
      if (cufftPlan3d(&h->plan_inv, N, N, N, CUFFT_Z2D) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, std::string(where) + ": cufftPlan3d failed");
      h->plan_inv_ok = true;
      if (cufftSetStream(h->plan_inv, h->stream) != CUFFT_SUCCESS) return h->fail(CLB_ECUDA, std::string(where) + ": cufftSetStream failed");
    }
    return CLB_OK;
  }

  // C2R of the half spectrum in buf (in place), scaled by 1/N^3, plus add, into dst.
  int to_space(double *buf, double *dst, double add)
  {
    if (cufftExecZ2D(h->plan_inv, reinterpret_cast<cufftDoubleComplex *>(buf), buf) != CUFFT_SUCCESS)
      return h->fail(CLB_ECUDA, std::string(where) + ": cufftExecZ2D failed");
    const double inv = 1.0 / ((double)N * (double)N * (double)N);
    CLB_LAUNCH(h, K_INIT, k_ic_extract<<<kICBlocks, 256, 0, h->stream>>>(buf, dst, N, inv, add));
    CLB_CHECK_LAUNCH(h, where);
    return CLB_OK;
  }

  int component(int kind, int comp, double m2c, double m20, double *F, double *P, double f0, double p0)
  {
    for (int which = 0; which < 2; ++which) {
      ModeArgs a = base;
      a.kind = kind;
      a.comp = comp;
      a.which = which;
      a.m2c = m2c;
      a.m20 = m20;
      CLB_LAUNCH(h, K_INIT, k_ic_modes<<<kICBlocks, 256, 0, h->stream>>>(reinterpret_cast<double2 *>(h->d_spec), a));
      CLB_CHECK_LAUNCH(h, where);
      const int r = to_space(h->d_spec, which == 0 ? F : P, which == 0 ? f0 : p0);
      if (r != CLB_OK) return r;
    }
    return CLB_OK;
  }

  // Gauss solve for the charge density of form: momenta out[3 * dir * stride] for dir = 0, 1, 2.
  int gauss(const double *F, const double *P, ChargeArgs ca, double *out, size_t stride)
  {
    CLB_LAUNCH(h, K_INIT, k_ic_charge<<<kICBlocks, 256, 0, h->stream>>>(F, P, h->d_spec, ca));
    CLB_CHECK_LAUNCH(h, where);
    if (cufftExecD2Z(h->plan, h->d_spec, reinterpret_cast<cufftDoubleComplex *>(h->d_spec)) != CUFFT_SUCCESS)
      return h->fail(CLB_ECUDA, std::string(where) + ": cufftExecD2Z failed");
    for (int dir = 0; dir < 3; ++dir) {
      CLB_LAUNCH(h, K_INIT, k_ic_gauss<<<kICBlocks, 256, 0, h->stream>>>(reinterpret_cast<const double2 *>(h->d_spec),
                                                                         reinterpret_cast<double2 *>(h->d_spec2), N, dir));
      CLB_CHECK_LAUNCH(h, where);
      const int r = to_space(h->d_spec2, out + (size_t)dir * stride, 0.0);
      if (r != CLB_OK) return r;
    }
    return CLB_OK;
  }

  // Volume means of nc components (deterministic: fixed-order block sums, then in order on the host).
  int means(const double *x, int nc, double *out, double *d_part)
  {
    std::vector<double> part(kICBlocks);
    for (int c = 0; c < nc; ++c) {
      CLB_LAUNCH(h, K_INIT, k_ic_sum<<<kICBlocks, 256, 0, h->stream>>>(x + (size_t)c * n3, n3, d_part));
      cudaError_t e = cudaMemcpyAsync(part.data(), d_part, kICBlocks * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess) return h->cuda_fail(e, where);
      double s = 0;
      for (double v : part) s += v;
      out[c] = s / (double)n3;
    }
    return CLB_OK;
  }
};

} // namespace

extern "C" int clb_generate_state(clb_handle *h, const clb_ic_params *p, const clb_scalefactor *sf)
{
  if (!h) return CLB_EINVAL;
  if (!p) return h->fail(CLB_EINVAL, "clb_generate_state: null parameters");
  if (!std::isfinite(p->amplitude) || !std::isfinite(p->k_cutoff) || !std::isfinite(p->adot))
    return h->fail(CLB_EINVAL, "clb_generate_state: amplitude, k_cutoff and adot must be finite");
  const int kind = h->md.kind;
  int NF, NP, nm;
  if (h->u1) {
    NF = NP = 5;
    nm = 2;
  } else if (h->su2) {
    NF = 22;
    NP = 19;
    nm = 7;
  } else {
    NF = NP = h->NS;
    nm = h->NS;
  }
  for (int c = 0; c < nm; ++c)
    if (!std::isfinite(p->mass2[c]) || !std::isfinite(p->fld0[c]) || !std::isfinite(p->pi0[c]))
      return h->fail(CLB_EINVAL, "clb_generate_state: non-finite mass2, fld0 or pi0");
  Gen g{h};
  g.N = h->N;
  g.n3 = h->n3;
  g.spec_n = (size_t)g.N * g.N * 2 * (g.N / 2 + 1);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_generate_state");
  int r = g.ensure_fft();
  if (r != CLB_OK) return r;
  double *F = nullptr, *P = nullptr, *d_part = nullptr;
  auto release = [&]() {
    cudaStreamSynchronize(h->stream);
    if (F) cudaFree(F);
    if (P) cudaFree(P);
    if (d_part) cudaFree(d_part);
  };
  if (cudaMalloc(&F, (size_t)NF * g.n3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&P, (size_t)NP * g.n3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&d_part, kICBlocks * sizeof(double)) != cudaSuccess) {
    release();
    return h->fail(CLB_ENOMEM, "clb_generate_state: the FP64 staging state does not fit");
  }
  const double dx = h->cfg.dx, L = g.N * dx;
  g.base.N = g.N;
  g.base.seed = p->seed;
  g.base.kIR = 2 * 3.14159265358979323846 / L;
  g.base.kcut = p->k_cutoff;
  g.base.A = p->amplitude * std::pow(L / (dx * dx), 1.5) / std::sqrt(2.0);
  g.base.adot = p->adot;
  const double fo = h->md.fStar / h->md.omegaStar, r2 = fo * fo;
  const double *m2 = p->mass2, *f0 = p->fld0, *q0 = p->pi0;
  const size_t n3 = g.n3;
  if (kind == CLB_MODEL_LPHI4) {
    for (int i = 0; i < NF && r == CLB_OK; ++i) r = g.component(0, i, m2[i], m2[i], F + i * n3, P + i * n3, f0[i], q0[i]);
  } else if (kind == CLB_MODEL_LPHI4U1) {
    for (int c = 0; c < 2 && r == CLB_OK; ++c) r = g.component(1, c, m2[c], m2[0], F + c * n3, P + c * n3, f0[c], q0[c]);
    if (r == CLB_OK && (e = cudaMemsetAsync(F + 2 * n3, 0, 3 * n3 * sizeof(double), h->stream)) != cudaSuccess)
      r = h->cuda_fail(e, "clb_generate_state");
    if (r == CLB_OK) r = g.gauss(F, P, ChargeArgs{g.N, 0, n3, dx, r2, p->charge[0], 0.0}, P + 2 * n3, n3);
  } else {
    // S; phi (1, 2); Phi (3-6); A = 0 (7-9); links = 1 (10 + 4 i); momenta: pi_A 7-9, pi_SU2 10 + 3 i + b
    if ((e = cudaMemsetAsync(F, 0, (size_t)NF * n3 * sizeof(double), h->stream)) != cudaSuccess) r = h->cuda_fail(e, "clb_generate_state");
    if (r == CLB_OK) r = g.component(0, 0, m2[0], m2[0], F, P, f0[0], q0[0]);
    for (int c = 0; c < 2 && r == CLB_OK; ++c)
      r = g.component(1, c, m2[1 + c], m2[1], F + (1 + c) * n3, P + (1 + c) * n3, f0[1 + c], q0[1 + c]);
    for (int c = 0; c < 4 && r == CLB_OK; ++c)
      r = g.component(2, c, m2[3 + c], m2[3], F + (3 + c) * n3, P + (3 + c) * n3, f0[3 + c], q0[3 + c]);
    for (int b = 0; b < 3 && r == CLB_OK; ++b)
      r = g.gauss(F, P, ChargeArgs{g.N, 1 + b, n3, dx, r2, p->charge[0], 0.0}, P + (10 + b) * n3, 3 * n3);
    if (r == CLB_OK) r = g.gauss(F, P, ChargeArgs{g.N, 4, n3, dx, r2, p->charge[1], p->charge[2]}, P + 7 * n3, n3);
    for (int i = 0; i < 3 && r == CLB_OK; ++i) {
      CLB_LAUNCH(h, K_INIT, k_ic_fill<<<kICBlocks, 256, 0, h->stream>>>(F + (10 + 4 * i) * n3, n3, 1.0));
      if ((e = cudaGetLastError()) != cudaSuccess) r = h->cuda_fail(e, "clb_generate_state");
    }
  }
  if (r == CLB_OK && (e = cudaStreamSynchronize(h->stream)) != cudaSuccess) r = h->cuda_fail(e, "clb_generate_state");
  if (r == CLB_OK) {
    if (h->u1) r = u1_set_state(h, F, P, sf);
    else if (h->su2) r = su2_set_state(h, F, P, sf);
    else {
      double mu[4] = {0, 0, 0, 0};
      if (h->fp32) {
        r = g.means(F, NF, mu, d_part);
        if (r == CLB_OK) r = g.means(P, NP, mu + 2, d_part);
      }
      if (r == CLB_OK) r = scalar_set_state(h, F, P, sf, h->fp32 ? mu : nullptr);
    }
  }
  collect_profile(h);
  release();
  return r;
}
