// clb_spectrum.cuh - radially binned power spectrum of one lattice component (cuFFT D2Z + binning).
//
// PowerSpectrumMeasurer::powerSpectrum (measurements/powerspectrum.h:84-134): |f_k|^2 of the
// unnormalised forward transform, projected radially over the full k-space.  The half spectrum
// (kz = 0 .. N/2) stands for the whole: each stored mode with 0 < kz < N/2 (or, for odd N, kz > 0)
// represents itself and its conjugate partner, so it counts twice; per-bin counts are then mode
// counts of the full N^3 grid.  Bin rule (TempLat's radial projector is not vendored; stated choice):
// b = floor(|n| / dk) with |n| the integer wave-vector norm; modes with b >= nbins fold into the last
// bin when `fold` is set, else they are left out.
#pragma once

#include "clb_internal.cuh"
#include "clb_sweep.cuh"

namespace clb {
// The non-template kernels are static: every unit that includes this header gets its own copies.

// Padded component -> real input of an in-place R2C transform (row pitch 2 (N/2 + 1) doubles).
template <class R>
static __global__ void __launch_bounds__(256) k_spec_gather(const R *__restrict__ src, double *__restrict__ dst, Pad pd, double off)
{
  const int N = pd.N;
  const long long pitch = 2LL * (N / 2 + 1);
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int x = (int)(r / N), y = (int)(r % N);
    const R *s = src + pd.at(x, y, 0);
    double *d = dst + r * pitch;
    for (int z = threadIdx.x; z < N; z += blockDim.x) d[z] = off + (double)s[z];
  }
}

// Unpadded N^3 component (x slowest) -> real input of an in-place R2C transform.
static __global__ void __launch_bounds__(256) k_spec_gather_plain(const double *__restrict__ src, double *__restrict__ dst, int N)
{
  const long long pitch = 2LL * (N / 2 + 1);
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const double *s = src + r * N;
    double *d = dst + r * pitch;
    for (int z = threadIdx.x; z < N; z += blockDim.x) d[z] = s[z];
  }
}

// Unpadded N^3 component of storage type R -> real input of an in-place R2C transform.
template <class R>
static __global__ void __launch_bounds__(256) k_spec_gather_raw(const R *__restrict__ src, double *__restrict__ dst, int N)
{
  const long long pitch = 2LL * (N / 2 + 1);
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const R *s = src + r * N;
    double *d = dst + r * pitch;
    for (int z = threadIdx.x; z < N; z += blockDim.x) d[z] = (double)s[z];
  }
}

// Tangent of the binned sum of |f_k|^2: per bin sum w 2 Re(conj(f_k) t_k) of the transforms of
// a component (fk) and of its tangent (tk), with k_spec_bin's bins and weights; partial rows in
// k_spec_bin's layout (the |n| and count slots left 0).
static __global__ void __launch_bounds__(256)
    k_spec_bin_cross(const double2 *__restrict__ fk, const double2 *__restrict__ tk, int N, double dk, int nbins,
                     int fold, double *__restrict__ part_val, unsigned long long *__restrict__ part_cnt)
{
  extern __shared__ unsigned char smem_raw[];
  double *h_val = reinterpret_cast<double *>(smem_raw);
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) h_val[b] = 0.0;
  __syncthreads();
  const int nzh = N / 2 + 1;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int kx = (int)(r / N), ky = (int)(r % N);
    const long long nx = kx <= N / 2 ? kx : kx - N;
    const long long ny = ky <= N / 2 ? ky : ky - N;
    const double2 *row = fk + r * nzh, *trow = tk + r * nzh;
    for (int kz = threadIdx.x; kz < nzh; kz += blockDim.x) {
      const long long n2 = nx * nx + ny * ny + (long long)kz * kz;
      const double nn = sqrt((double)n2);
      int b = (int)floor(nn / dk);
      if (b >= nbins) {
        if (!fold) continue;
        b = nbins - 1;
      }
      const int w = (kz == 0 || (2 * kz == N)) ? 1 : 2;
      const double2 v = row[kz], t = trow[kz];
      atomicAdd(&h_val[b], w * (2.0 * (v.x * t.x + v.y * t.y)));
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
    part_val[((size_t)blockIdx.x * nbins + b) * 2 + 0] = h_val[b];
    part_val[((size_t)blockIdx.x * nbins + b) * 2 + 1] = 0.0;
    part_cnt[(size_t)blockIdx.x * nbins + b] = 0ull;
  }
}

// Gradient of sum_b g_b (sum over bin b of |f_k|^2), step 1: each mode of the half spectrum times
// the weight g of its bin (k_spec_bin's bin rule; modes outside the bins: 0).  A C2R transform of
// the result, times 2, is the gradient with respect to the real component.
static __global__ void __launch_bounds__(256)
    k_spec_weight(double2 *__restrict__ fk, int N, double dk, int nbins, int fold, const double *__restrict__ gbin)
{
  const int nzh = N / 2 + 1;
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const int kx = (int)(r / N), ky = (int)(r % N);
    const long long nx = kx <= N / 2 ? kx : kx - N;
    const long long ny = ky <= N / 2 ? ky : ky - N;
    double2 *row = fk + r * nzh;
    for (int kz = threadIdx.x; kz < nzh; kz += blockDim.x) {
      const long long n2 = nx * nx + ny * ny + (long long)kz * kz;
      int b = (int)floor(sqrt((double)n2) / dk);
      double g = 0.0;
      if (b < nbins || fold) g = gbin[b < nbins ? b : nbins - 1];
      row[kz] = double2{row[kz].x * g, row[kz].y * g};
    }
  }
}

// Real output of an in-place C2R transform (row pitch 2 (N/2 + 1)) times scale -> N^3 array.
static __global__ void __launch_bounds__(256) k_spec_extract(const double *__restrict__ src, double *__restrict__ dst, int N, double scale)
{
  const long long pitch = 2LL * (N / 2 + 1);
  for (long long r = blockIdx.x; r < (long long)N * N; r += gridDim.x) {
    const double *s = src + r * pitch;
    double *d = dst + r * N;
    for (int z = threadIdx.x; z < N; z += blockDim.x) d[z] = scale * s[z];
  }
}

// One block per group of (kx, ky) rows; shared-memory histograms of sum w |f|^2, sum w |n| and the
// integer mode count, written as one partial row per block.
static __global__ void __launch_bounds__(256)
    k_spec_bin(const double2 *__restrict__ fk, int N, double dk, int nbins, int fold, double *__restrict__ part_val,
               unsigned long long *__restrict__ part_cnt)
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
    const long long nx = kx <= N / 2 ? kx : kx - N;
    const long long ny = ky <= N / 2 ? ky : ky - N;
    const double2 *row = fk + r * nzh;
    for (int kz = threadIdx.x; kz < nzh; kz += blockDim.x) {
      const long long n2 = nx * nx + ny * ny + (long long)kz * kz;
      const double nn = sqrt((double)n2);
      int b = (int)floor(nn / dk);
      if (b >= nbins) {
        if (!fold) continue;
        b = nbins - 1;
      }
      const int w = (kz == 0 || (2 * kz == N)) ? 1 : 2;
      const double2 v = row[kz];
      const double p = v.x * v.x + v.y * v.y;
      atomicAdd(&h_val[b], w * p);
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

// Fixed-order sum of the block partial rows, one thread per bin.
static __global__ void __launch_bounds__(256)
    k_spec_sum(const double *__restrict__ part_val, const unsigned long long *__restrict__ part_cnt, int nblk, int nbins,
               double *__restrict__ out_val, double *__restrict__ out_n, unsigned long long *__restrict__ out_cnt)
{
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  double v = 0, n = 0;
  unsigned long long c = 0;
  for (int k = 0; k < nblk; ++k) {
    v += part_val[((size_t)k * nbins + b) * 2 + 0];
    n += part_val[((size_t)k * nbins + b) * 2 + 1];
    c += part_cnt[(size_t)k * nbins + b];
  }
  out_val[b] = v;
  out_n[b] = n;
  out_cnt[b] = c;
}

} // namespace clb
