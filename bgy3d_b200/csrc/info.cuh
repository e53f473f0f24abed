// info.cuh -- post-processing observables of a solute solve: info() /
// print_info() (bgy3d-potential.c:245-493) and the grid moments of
// bgy3d_moments (bgy3d-vec.c:476-593).
//
//   rho_v = rho sum_i q_i g_i            solvent charge density
//   v_e   = Poisson potential of rho_v   (bgy3d_poisson, bgy3d-poisson.c:103-183:
//                                         4 pi/eps0 rho_v(k)/k^2, zero mean)
//   rho_u = (G/sqrt pi)^3 sum q e^{-G^2 r^2}  Gaussian cores (bgy3d-solutes.c:555-577)
//   u_c   = long-range solute Coulomb     (coulomb_long, bgy3d-solutes.c:795-815)
//
// <U_v|rho_u> = h^3 sum v_e rho_u is taken in k space (Parseval over the
// r2c half spectrum), and v_e at arbitrary points by the trigonometric sum of
// bgy3d_fft_interp (bgy3d-fftw3.c:504-612) over the same spectrum -- at the
// solute sites, and at the 8 grid nodes around each site for the trilinear
// value of bgy3d_interp (bgy3d-interp.c:37-136).
#pragma once
#include "kernels.cuh"

namespace rism {

// Block partials of the moments of shift + scale * v for `nf` fields of the
// grid: part[(f * gridDim.x + block) * 10 + {sum, x, y, z, xx, yy, zz, xy,
// yz, zx}] with x = i0 - N0/2 etc. (vec_moments1/2 take the grid index
// about 0.5 N, not the box centre).
static __global__ void __launch_bounds__(256) k_moments(Geo g, const double *__restrict__ v, int nf, double shift,
                                                        double scale, double *__restrict__ part) {
  const int f = blockIdx.y;
  double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double *vf = v + (long long)f * g.Nr;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.Nr;
       p += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(p % g.N0);
    const int i1 = (int)((p / g.N0) % g.N1);
    const int i2 = (int)(p / ((long long)g.N0 * g.N1));
    const double x = i0 - 0.5 * g.N0, y = i1 - 0.5 * g.N1, z = i2 - 0.5 * g.N2;
    const double w = shift + scale * vf[p];
    acc[0] += w;
    acc[1] += w * x;
    acc[2] += w * y;
    acc[3] += w * z;
    acc[4] += w * x * x;
    acc[5] += w * y * y;
    acc[6] += w * z * z;
    acc[7] += w * x * y;
    acc[8] += w * y * z;
    acc[9] += w * z * x;
  }
  __shared__ double sm[10][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    double a = acc[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) sm[k][wid] = a;
  }
  __syncthreads();
  if (threadIdx.x < 10) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sm[threadIdx.x][w];
    part[((long long)f * gridDim.x + blockIdx.x) * 10 + threadIdx.x] = a;
  }
}

// rho_v = rho sum_i q_i g_i with g = 1 + h from T (closure at v); rho_u the
// Gaussian cores; written into out[0] and out[1] (two fields of Nr).
static __global__ void k_densities(Geo g, int m, const double *__restrict__ t, const double *__restrict__ v,
                                   double beta, int closure, const double *__restrict__ charge, double rho,
                                   double h0, double h1, double h2, double L0, double L1, double L2, int n,
                                   const SiteP *__restrict__ solute, double *__restrict__ rv,
                                   double *__restrict__ ru) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  double s = 0.0;
  for (int i = 0; i < m; ++i) {
    const long long o = (long long)i * g.Nr + p;
    const double ts = t[o];
    const double h = closure_c<double>(closure, beta * v[o], ts) + ts;
    s += charge[i] * rho * (h + 1.0);
  }
  rv[p] = s;
  const int i0 = (int)(p % g.N0);
  const int i1 = (int)((p / g.N0) % g.N1);
  const int i2 = (int)(p / ((long long)g.N0 * g.N1));
  const double x = i0 * h0 - L0 / 2, y = i1 * h1 - L1 / 2, z = i2 * h2 - L2 / 2;
  double c = 0.0;
  for (int u = 0; u < n; ++u) {
    const SiteP b = solute[u];
    const double r2 = (x - b.x) * (x - b.x) + (y - b.y) * (y - b.y) + (z - b.z) * (z - b.z);
    c += b.charge * exp(-(kG * kG) * r2);
  }
  const double gs = kG / sqrt(M_PI);
  ru[p] = (gs * gs * gs) * c;
}

// The solvent potential's spectrum V(k) = 4 pi/eps0 Rv(k)/k^2 (0 at k = 0)
// from the forward transform Rv of rho_v; the r2c half grid, W layout.
__device__ __forceinline__ double2 poisson_k(const Geo &g, const double2 *__restrict__ Rv, int ix, int iy, int iz,
                                             long long o) {
  const double k0 = kfreq(ix, g.N0) * g.dk0, k1 = kfreq(iy, g.N1) * g.dk1, k2 = kfreq(iz, g.N2) * g.dk2;
  const double kq = k2 * k2 + k1 * k1 + k0 * k0;
  const double fac = kq != 0.0 ? 4 * M_PI * kEps0Inv / kq : 0.0;
  const double2 r = Rv[o];
  return make_double2(fac * r.x, fac * r.y);
}

// Block partials of the trigonometric interpolation of v_e at the points
// pts[blockIdx.y] (fractional grid coordinates) and, for blockIdx.y ==
// npts, of the Parseval sum w Re(V conj Ru) (w = 1 on the kx = 0 and
// kx = N0/2 planes, else 2); part[(y * gridDim.x + block)] before 1/N.
static __global__ void __launch_bounds__(256) k_info_kspace(Geo g, const double2 *__restrict__ Rv,
                                                            const double2 *__restrict__ Ru, int npts,
                                                            const double3 *__restrict__ pts,
                                                            double *__restrict__ part) {
  const int q = blockIdx.y;
  const long long tot = (long long)g.Nh * g.N1 * g.N2;
  double acc = 0.0;
  double3 x = make_double3(0, 0, 0);
  if (q < npts) x = pts[q];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < tot;
       p += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(p % g.Nh);
    const int iy = (int)((p / g.Nh) % g.N1);
    const int iz = (int)(p / ((long long)g.Nh * g.N1));
    const long long o = ((long long)iz * g.N1 + iy) * g.Nhp + ix;
    const double2 V = poisson_k(g, Rv, ix, iy, iz, o);
    if (q == npts) {
      const double2 u = Ru[o];
      const double w = (ix == 0 || ix == g.M) ? 1.0 : 2.0;
      acc += w * (V.x * u.x + V.y * u.y);
      continue;
    }
    // waves: e^{i 2 pi K x / N}, cos on the self-conjugate indices
    double wr = 1.0, wi = 0.0;
    const int idx[3] = {ix, iy, iz}, NN[3] = {g.N0, g.N1, g.N2};
    const double xx[3] = {x.x, x.y, x.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int K = kfreq(idx[d], NN[d]);
      const double ph = (2 * M_PI / NN[d]) * K * xx[d];
      double s, c;
      sincos(ph, &s, &c);
      if ((NN[d] - 2 * idx[d]) % NN[d] == 0) s = 0.0;
      const double nr = wr * c - wi * s, ni = wr * s + wi * c;
      wr = nr;
      wi = ni;
    }
    const double half = ((g.N0 - 2 * ix) % g.N0 == 0) ? 0.5 : 1.0;
    acc += 2.0 * half * (V.x * wr - V.y * wi);
  }
  __shared__ double sm[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) sm[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sm[w];
    part[(long long)q * gridDim.x + blockIdx.x] = a;
  }
}

// Block partials of sum u_c rho_v (for <rho_v|U_u>).
static __global__ void __launch_bounds__(256) k_dot(long long n, const double *__restrict__ a,
                                                    const double *__restrict__ b, double *__restrict__ part) {
  double acc = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
    acc += a[p] * b[p];
  __shared__ double sm[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) sm[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[w];
    part[blockIdx.x] = s;
  }
}

}  // namespace rism
