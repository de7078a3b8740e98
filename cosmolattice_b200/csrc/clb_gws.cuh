// clb_gws.cuh - storage of the gravitational-wave sector and the kick and drift kernels that every
// model's GWs share; only the source differs (clb_gws.cu: the scalar singlets; clb_u1.cu: lphi4U1;
// clb_su2.cu: lphi4SU2U1).
//
// u_ij is stored as five components (u_11, u_12, u_13, u_22, u_23; u_33 = -u_11 - u_22, the storage
// gwsprojector.h reads) of N^3 sites each, x slowest.  The kick (GWsKernels::get, gwskernels.h:27-33,
// applied by LeapFrog::kickGWs) is
//   pi_u += h [a^(1+alpha) lapl(u) + a^(1+alpha) 2 Pi],
// with lapl the seven-point Laplacian of each component (gaugederivatives.h:42-46) and Pi the
// traceless part (Pi_11 - tr/3, Pi_12, Pi_13, Pi_22 - tr/3, Pi_23) of the anisotropic tensor
// (PITensor.h:52-57) that the source forms at the site.  The drift (LeapFrog::driftGWs) is
// u += pow(a_SI, alpha - 3) (dt pi_u).  FP64 pins every rounding (Ar<double>, divisions rounded).
#pragma once

#include "clb_internal.cuh"
#include "clb_scalar.cuh"

namespace clb {

struct GWSector {
  void *u = nullptr, *pi = nullptr; // 5 x N^3 each, the storage type of the handle's fields
  bool fp32 = false;                 // FP32 storage and arithmetic (the handle's FP32 form)
  bool synced = true;                // momenta at integer time (after clb_initialize or a sync)
  double *d_fk = nullptr;            // five in-place D2Z buffers of the spectrum
};

constexpr int kGWBlocks = 148 * 8;

// Tensor index k of the pair (i, j), i <= j: 00, 01, 02, 11, 12, 22.
__host__ __device__ constexpr int gw_pair_i(int k) { return k < 3 ? 0 : k < 5 ? 1 : 2; }
__host__ __device__ constexpr int gw_pair_j(int k) { return k < 3 ? k : k < 5 ? k - 2 : 2; }

// pi_u += h K(u; a_I) at every site, the source src(s, x, y, z, xp, yp, zp, P) giving the
// anisotropic tensor P at site s = (x, y, z) (xp, yp, zp: its forward neighbours' coordinates);
// kA points at the device copy of pow(a_I, 1 + alpha).
template <class R, class Src>
__global__ void __launch_bounds__(256) k_gw_kick(const R *__restrict__ u, R *__restrict__ piu, int N, double inv_dx2d,
                                                 double hd, const double *__restrict__ kA_ptr, Src src)
{
  using A = Ar<R>;
  const size_t n3 = (size_t)N * N * N;
  const R kA = (R)*kA_ptr, h = (R)hd, inv_dx2 = (R)inv_dx2d, two = R(2), third = R(1.0 / 3.0);
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(s % N), y = (int)((s / N) % N), x = (int)(s / ((size_t)N * N));
    const int xp = x + 1 == N ? 0 : x + 1, xm = x == 0 ? N - 1 : x - 1;
    const int yp = y + 1 == N ? 0 : y + 1, ym = y == 0 ? N - 1 : y - 1;
    const int zp = z + 1 == N ? 0 : z + 1, zm = z == 0 ? N - 1 : z - 1;
    R P[6];
    src(s, x, y, z, xp, yp, zp, P);
    const R tr3 = A::mul(A::add(A::add(P[0], P[3]), P[5]), third);
    const R S[5] = {A::sub(P[0], tr3), P[1], P[2], A::sub(P[3], tr3), P[4]};
    const R kA2 = A::mul(kA, two);
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const R *U = u + (size_t)c * n3;
      const R uc = U[s];
      const R tx = A::sub(A::add(U[((size_t)xp * N + y) * N + z], U[((size_t)xm * N + y) * N + z]), A::mul(two, uc));
      const R ty = A::sub(A::add(U[((size_t)x * N + yp) * N + z], U[((size_t)x * N + ym) * N + z]), A::mul(two, uc));
      const R tz = A::sub(A::add(U[((size_t)x * N + y) * N + zp], U[((size_t)x * N + y) * N + zm]), A::mul(two, uc));
      const R lap = A::mul(inv_dx2, A::add(A::add(tx, ty), tz));
      const R K = A::add(A::mul(kA, lap), A::mul(kA2, S[c]));
      piu[(size_t)c * n3 + s] = A::add(piu[(size_t)c * n3 + s], A::mul(h, K));
    }
  }
}

// u += pow(a_SI, alpha - 3) (dt pi_u); pd points at the device copy of pow(a_SI, alpha - 3).
template <class R>
__global__ void __launch_bounds__(256) k_gw_drift(R *__restrict__ u, const R *__restrict__ piu, size_t n, double dtd,
                                                  const double *__restrict__ pd_ptr)
{
  const R pd = (R)*pd_ptr, dt = (R)dtd;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    u[i] = drift_val<R>(u[i], piu[i], pd, dt);
}

// The same drift with the coefficient formed here from a_SI (aSI points at the device copy; the
// position-Verlet tails keep a_SI as the reference does, positionverlet.h:213-235, but their drift
// coefficient is a_I's).
template <class R>
__global__ void __launch_bounds__(256) k_gw_drift_a(R *__restrict__ u, const R *__restrict__ piu, size_t n, double dtd,
                                                    const double *__restrict__ aSI, double alpha)
{
  const R pd = (R)apow(*aSI, alpha - 3), dt = (R)dtd;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    u[i] = drift_val<R>(u[i], piu[i], pd, dt);
}

// Launches the GW drift: with the tails' coefficient pd (VV, leapfrog), or from a_SI (position Verlet).
template <class R>
inline void launch_gw_drift(R *u, const R *piu, size_t n, double dt, const double *pd, const double *aSI, double alpha,
                            bool from_aSI, cudaStream_t stream)
{
  if (from_aSI)
    k_gw_drift_a<R><<<kGWBlocks, 256, 0, stream>>>(u, piu, n, dt, aSI, alpha);
  else
    k_gw_drift<R><<<kGWBlocks, 256, 0, stream>>>(u, piu, n, dt, pd);
}

// The gauge part of the anisotropic tensor (PITensor.h:58-111) at site s, added to P in the
// reference's order: P_ij += 2 Re[D_i phi conj(D_j phi)] (complex scalar), then the U(1) electric
// and magnetic terms -1/a^2/(fStar/omegaStar)^2 pi_A,i pi_A,j and ... B_i B_j.  phi (fr, fi at the
// components' bases) couples to A through the link complexPhase(ndxg A_i) with ndxg = (-dx) gQ;
// D_i phi = (U_i(x) phi(x + i) - phi(x)) / dx (forwardCovGradientCS, gaugederivatives.h:75-78);
// B = (F_23, F_31, F_12) with F(A, i, j) = forwDiff(A_j, i) - forwDiff(A_i, j) (a stated choice of
// TempLat's fieldStrength; the products B_i B_j do not depend on its sign).  first: P holds no
// singlet part yet, so the complex term starts it.
template <class R>
__device__ __forceinline__ void gw_gauge_tensor(const R *__restrict__ phr, const R *__restrict__ phi,
                                                const R *__restrict__ Ax, const R *__restrict__ pAx, size_t n3,
                                                const size_t (&nb)[3], size_t s, R dx, R ndxg, R aI, R rfo2, bool first,
                                                R (&P)[6])
{
  using A = Ar<R>;
  const R fr = phr[s], fi = phi[s];
  R dr[3], di[3], B[3], E[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const R th = A::mul(ndxg, Ax[(size_t)i * n3 + s]);
    const R ur = cos(th), ui = sin(th);
    const R pr = phr[nb[i]], pm = phi[nb[i]];
    const R wr = A::sub(A::mul(ur, pr), A::mul(ui, pm)), wi = A::add(A::mul(ur, pm), A::mul(ui, pr));
    dr[i] = A::sub(wr, fr) / dx;
    di[i] = A::sub(wi, fi) / dx;
    E[i] = pAx[(size_t)i * n3 + s];
  }
  // forwDiff(A_j, i)
  auto fdA = [&](int j, int i) { return A::sub(Ax[(size_t)j * n3 + nb[i]], Ax[(size_t)j * n3 + s]) / dx; };
  B[0] = A::sub(fdA(2, 1), fdA(1, 2));
  B[1] = A::sub(fdA(0, 2), fdA(2, 0));
  B[2] = A::sub(fdA(1, 0), fdA(0, 1));
  const R pref = (R(-1) / A::mul(aI, aI)) / rfo2;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int i = gw_pair_i(k), j = gw_pair_j(k);
    const R c = A::mul(R(2), A::add(A::mul(dr[i], dr[j]), A::mul(di[i], di[j])));
    const R e = A::mul(A::mul(pref, E[i]), E[j]);
    const R m = A::mul(A::mul(pref, B[i]), B[j]);
    P[k] = A::add(A::add(first ? c : A::add(P[k], c), e), m);
  }
}

} // namespace clb
