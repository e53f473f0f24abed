// grad.cuh -- kernels of the free-energy gradient dmu/d(solute q, sigma,
// eps, R) by the adjoint of the converged fixed point (renormalised form).
//
// mu = (rho h^3 / beta) sum_i sum_r f(x_i, h_i, c_i, cl_i), the closure's
// free-energy density form() with x = -beta v + t, c = c(x) - t, h = c + t,
// cl = -beta q_i uc (closures.f90:574-612, hnc3d.c:2157-2269).  With the
// adjoint J^T lambda = d mu / d t at the root F(t) = 0,
//
//   dmu/dp = sum_r sum_i A_i dv_i/dp + sum_r B duc/dp  +  tau term,
//   A_i = (rho h^3/beta) df/dv + beta (K lambda)_i (c'_i + 1),
//   B   = rho h^3 sum_i q_i h_i / 2,
//
// K = (chi - 1) * the OZ convolution (symmetric) and c' = dc/dt; the tau
// term is the renormalised long-range field's share,
// (1/N) sum_i sum_k w_k Re[S_i(k) dL(k)/dp conj(FFT lambda_i)(k)] over the
// half spectrum (w_k = 1 on the kx = 0 and kx = N0/2 planes, else 2).
// The solute field and its derivatives follow field0 / field1
// (bgy3d-solutes.c:343-468) with the capped LJ and short-range Coulomb
// (bgy3d-solutes.c:101-114, 230-243) and the long-range uc (795-815).
#pragma once
#include "kernels.cuh"

namespace rism {

// Partial derivatives of form(method, x, h, c, cl) in its arguments.
__device__ __forceinline__ void form_partials(int method, double x, double h, double c, double cl, double &fx,
                                              double &fh, double &fc, double &fcl) {
  fc = -1.0 - h / 2;
  fh = -(c + cl) / 2;
  fcl = -h / 2;
  fx = 0.0;
  switch (method) {
    case CL_HNC: fh += h; break;
    case CL_KH: if (h < 0) fh += h; break;
    case CL_PY: break;
    default: {
      fh += h;
      if (h >= 0) {  // - x^mm / mm!  ->  - x^(mm-1) / (mm-1)!
        const int mm = method - CL_PSE0 + 1;
        double xm = 1.0;
        for (int k = 0; k < mm - 1; ++k) xm *= x;
        fx = -xm / dfact(mm - 1);
      }
    }
  }
}

// r-derivatives divided by r of the capped pair functions (finite at r = 0).
__device__ __forceinline__ double ljcap1(double s) {  // d ljcap0 / ds
  const double R = 0.2;
  if (s >= R) return lj1(s);
  return 2 * (lj1(R) / (2 * R)) * s;
}
__device__ __forceinline__ double ljcap1s(double s) {  // ljcap1(s) / s
  const double R = 0.2;
  if (s >= R) return lj1(s) / s;
  return lj1(R) / R;
}
__device__ __forceinline__ double cscap1s(double r) {  // (d cscap0 / dr) / r
  const double R = 0.2;
  if (r >= R) return cs1(r) / r;
  return cs1(R) / R;
}
__device__ __forceinline__ double cl1s(double r) {  // (d cl0 / dr) / r
  if (r >= 0.02) return ((2 / sqrt(M_PI)) * r * exp(-r * r) - erf(r)) / (r * r * r);
  const double r2 = r * r;
  return (2 / sqrt(M_PI)) * (-2. / 3. + r2 * (4. / 10. + r2 * (-6. / 42.)));
}

// b_i = d mu / d t_i = (rho h^3/beta) (f_c c' + f_h (c' + 1) + f_x).
static __global__ void k_mu_dt(Geo g, const double *__restrict__ t, const double *__restrict__ v,
                               const double *__restrict__ uc, double beta, int closure,
                               const double *__restrict__ charge, double rhoh3b, double *__restrict__ b) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  for (int s = 0; s < g.m; ++s) {
    const long long o = (long long)s * g.Nr + p;
    const double ts = t[o], bv = beta * v[o];
    const double c = closure_c<double>(closure, bv, ts), d = closure_d<double>(closure, bv, ts);
    const double h = c + ts, x = -bv + ts, cl = -beta * charge[s] * uc[p];
    double fx, fh, fc, fcl;
    form_partials(closure, x, h, c, cl, fx, fh, fc, fcl);
    b[o] = rhoh3b * (fc * d + fh * (d + 1) + fx);
  }
}

// A_i (m fields) and B (one field) of the gradient sums; kl = K lambda.
static __global__ void k_grad_weights(Geo g, const double *__restrict__ t, const double *__restrict__ v,
                                      const double *__restrict__ uc, const double *__restrict__ kl, double beta,
                                      int closure, const double *__restrict__ charge, double rhoh3b, double rhoh3,
                                      double *__restrict__ A, double *__restrict__ B) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  double bsum = 0.0;
  for (int s = 0; s < g.m; ++s) {
    const long long o = (long long)s * g.Nr + p;
    const double ts = t[o], bv = beta * v[o];
    const double c = closure_c<double>(closure, bv, ts), d = closure_d<double>(closure, bv, ts);
    const double h = c + ts, x = -bv + ts, cl = -beta * charge[s] * uc[p];
    double fx, fh, fc, fcl;
    form_partials(closure, x, h, c, cl, fx, fh, fc, fcl);
    const double fv = -beta * ((fc + fh) * (d + 1) + fx);
    A[o] = rhoh3b * fv + beta * kl[o] * (d + 1);
    bsum += charge[s] * h / 2;
  }
  B[p] = rhoh3 * bsum;
}

// Real-space sums for solute site u = blockIdx.y over this block's grid
// points: part[(u * gridDim.x + blockIdx.x) * 6 + {q, sigma, eps, x, y, z}].
static __global__ void __launch_bounds__(256) k_grad_real(Geo g, double h0, double h1, double h2, double L0,
                                                          double L1, double L2, const SiteP *__restrict__ solvent,
                                                          const SiteP *__restrict__ solute,
                                                          const double *__restrict__ A, const double *__restrict__ B,
                                                          double *__restrict__ part) {
  const int u = blockIdx.y;
  const SiteP su = solute[u];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.Nr;
       p += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(p % g.N0);
    const int i1 = (int)((p / g.N0) % g.N1);
    const int i2 = (int)(p / ((long long)g.N0 * g.N1));
    const double dx = i0 * h0 - L0 / 2 - su.x, dy = i1 * h1 - L1 / 2 - su.y, dz = i2 * h2 - L2 / 2 - su.z;
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    double gr = 0.0;  // (1/r) d/dr of sum_i A_i v_iu
    for (int s = 0; s < g.m; ++s) {
      const SiteP a = solvent[s];
      const double w = A[(long long)s * g.Nr + p];
      const double eab = sqrt(a.epsilon * su.epsilon), sab = 0.5 * (a.sigma + su.sigma);
      const double sv = r / sab;
      const double qq = a.charge * kEps0Inv;  // times q_u: short-range Coulomb prefactor
      acc[0] += w * qq * kG * cscap0(kG * r);
      acc[1] += w * eab * ljcap1(sv) * (-sv / sab) * 0.5;
      if (eab > 0) acc[2] += w * (a.epsilon / (2 * eab)) * ljcap0(sv);
      gr += w * (eab * ljcap1s(sv) / (sab * sab) + qq * su.charge * kG * kG * kG * cscap1s(kG * r));
    }
    const double bw = B[p];
    acc[0] += bw * kEps0Inv * kG * cl0(kG * r);
    gr += bw * kEps0Inv * su.charge * kG * kG * kG * cl1s(kG * r);
    // d/dR_u = -(r - R_u) / r d/dr
    acc[3] -= gr * dx;
    acc[4] -= gr * dy;
    acc[5] -= gr * dz;
  }
  __shared__ double sm[6][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double a = acc[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) sm[k][wid] = a;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sm[threadIdx.x][w];
    part[((long long)u * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = a;
  }
}

// k-space (tau) sums for solute site u = blockIdx.y over the half spectrum:
// Q(k) = sum_i S_i(|k|) conj(Lam_i(k)) with Lam = FFT lambda (in W) and S the
// radial tables of the long-range field (beta/eps0 s_i, value + slope
// pairs); part[(u * gridDim.x + b) * 4 + {q, x, y, z}] without the final
// 1/(N h^3).
static __global__ void __launch_bounds__(256) k_grad_kspace(Geo g, const double2 *__restrict__ Lam,
                                                            const double2 *__restrict__ stab, int nrad, double dkr,
                                                            const SiteP *__restrict__ solute,
                                                            double *__restrict__ part) {
  const int u = blockIdx.y;
  const SiteP su = solute[u];
  const long long tot = (long long)g.Nh * g.N1 * g.N2;
  double acc[4] = {0, 0, 0, 0};
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < tot;
       p += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(p % g.Nh);
    const int iy = (int)((p / g.Nh) % g.N1);
    const int iz = (int)(p / ((long long)g.Nh * g.N1));
    const int fx = kfreq(ix, g.N0), fy = kfreq(iy, g.N1), fz = kfreq(iz, g.N2);
    const double k0 = fx * g.dk0, k1 = fy * g.dk1, k2 = fz * g.dk2;
    const double kk = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)), __dmul_rn(k2, k2)));
    const double fi = kk / dkr - 0.5;
    int i = (int)(fi + 0.5);
    i = min(max(i, 0), nrad - 1);
    const double fr = fi - i;
    const long long o = ((long long)iz * g.N1 + iy) * g.Nhp + ix;
    double qr = 0.0, qi = 0.0;
    for (int s = 0; s < g.m; ++s) {
      const double2 sv = stab[(long long)s * nrad + i];
      const double S = sv.x + sv.y * fr;
      const double2 l = Lam[(long long)s * g.Nc + o];
      qr += S * l.x;
      qi -= S * l.y;
    }
    const int sgn = (((fx % 2) != 0) ^ ((fy % 2) != 0) ^ ((fz % 2) != 0)) ? -1 : 1;
    const double w = (ix == 0 || ix == g.M) ? 1.0 : 2.0;
    double sn, cs;
    sincos((k0 * su.x + k1 * su.y) + k2 * su.z, &sn, &cs);
    const double er = cs * qr + sn * qi, ei = cs * qi - sn * qr;  // e^{-i k.R} Q
    const double f = w * sgn;
    acc[0] += f * er;
    acc[1] += f * su.charge * k0 * ei;
    acc[2] += f * su.charge * k1 * ei;
    acc[3] += f * su.charge * k2 * ei;
  }
  __shared__ double sm[4][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double a = acc[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) sm[k][wid] = a;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sm[threadIdx.x][w];
    part[((long long)u * gridDim.x + blockIdx.x) * 4 + threadIdx.x] = a;
  }
}

static __global__ void k_fill(long long n, double v, double *__restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = v;
}

// out = d * a - b (the transposed Jacobian's epilogue: J^T v = d K v - v).
static __global__ void k_dmul_sub(long long n, const double *__restrict__ d, const double *__restrict__ a,
                                  const double *__restrict__ b, double *__restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = d[i] * a[i] - b[i];
}


// ---------------------------------------------------------- linear response
// dmu/dR by forward-mode linear response (the response branch of
// hnc3d_solute_solve, hnc3d.c:1969-2135, with response_t1, 1366-1421): per
// unit displacement of one solute site, dv = field1 (LJ plus the FULL capped
// Coulomb, bgy3d-solutes.c:381-468), J dT = beta K ((c' + 1) dv), and the
// differential of the free-energy density form1 (closures.f90:615-653).

// d ccap0 / dr, the capped full Coulomb 1/r (bgy3d-solutes.c:275-283): -1/r^2
// beyond R, the capped short-range plus long-range parts inside.
__device__ __forceinline__ double ccap1(double r) {
  const double R = 0.2;
  if (r >= R) return -1.0 / (r * r);
  return r * (cs1(R) / R + cl1s(r));
}

// Differential of form(method, x, h, c, cl) (closures.f90:615-653).
__device__ __forceinline__ double form1(int method, double x, double dx, double h, double dh, double c, double dc,
                                        double cl) {
  const double base = -dc - dh * (c + cl) / 2 - h * dc / 2;
  switch (method) {
    case CL_HNC: return base + h * dh;
    case CL_KH: return h < 0 ? base + h * dh : base;
    case CL_PY: return base;
    default: {
      if (h < 0) return base + h * dh;
      const int n = method - CL_PSE0;
      double xn = 1.0;
      for (int k = 0; k < n; ++k) xn *= x;
      return base + (h * dh - xn * dx / dfact(n));
    }
  }
}

// dv[s] = d v_s / d R_{u,dim} on the grid (field1 for one moving site).
static __global__ void k_field1(Geo g, double h0, double h1, double h2, double L0, double L1, double L2,
                                const SiteP *__restrict__ solvent, const SiteP *__restrict__ solute, int u, int dim,
                                double *__restrict__ dv) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  const int i0 = (int)(p % g.N0);
  const int i1 = (int)((p / g.N0) % g.N1);
  const int i2 = (int)(p / ((long long)g.N0 * g.N1));
  const SiteP b = solute[u];
  const double ab[3] = {i0 * h0 - L0 / 2 - b.x, i1 * h1 - L1 / 2 - b.y, i2 * h2 - L2 / 2 - b.z};
  const double r = sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
  const double dr = r > 0.0 ? -ab[dim] / r : 0.0;
  for (int s = 0; s < g.m; ++s) {
    const SiteP a = solvent[s];
    const double eab = sqrt(a.epsilon * b.epsilon), sab = 0.5 * (a.sigma + b.sigma);
    const double qab = a.charge * b.charge * kEps0Inv;
    dv[(long long)s * g.Nr + p] = dr * ((eab / sab) * ljcap1(r / sab) + qab * kG * kG * ccap1(kG * r));
  }
}

// The reference's free-energy gradient, the `derivatives` output of
// hnc3d_solute_solve (gradients / energy1, hnc3d.c:1665-1742, with field1,
// bgy3d-solutes.c:381-468): de[u][dim] = rho h^3 sum_i sum_r g_i(r)
// dv_i/dR_{u,dim}(r), g = c(t) + t + 1 and dv the LJ and FULL capped
// Coulomb derivative of a unit displacement of site u (0 at r = 0, where
// the reference takes no limit).  Block (blockIdx.x, blockIdx.y) sums sites
// u = U blockIdx.y ... U blockIdx.y + U - 1 over its grid points:
// part[(u * gridDim.x + blockIdx.x) * 3 + dim] (rho h^3 applied on the host).
template <int U>
static __global__ void __launch_bounds__(256) k_force_pair(Geo g, double h0, double h1, double h2, double L0,
                                                           double L1, double L2, const SiteP *__restrict__ solvent,
                                                           int n, const SiteP *__restrict__ solute,
                                                           const double *__restrict__ t,
                                                           const double *__restrict__ v, double beta, int closure,
                                                           double *__restrict__ part) {
  const int u0 = blockIdx.y * U;
  const int m = g.m;
  double acc[U][3];
#pragma unroll
  for (int k = 0; k < U; ++k) acc[k][0] = acc[k][1] = acc[k][2] = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.Nr;
       p += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(p % g.N0);
    const int i1 = (int)((p / g.N0) % g.N1);
    const int i2 = (int)(p / ((long long)g.N0 * g.N1));
    const double x = i0 * h0 - L0 / 2, y = i1 * h1 - L1 / 2, z = i2 * h2 - L2 / 2;
    double gs[kMaxSites];
#pragma unroll
    for (int s = 0; s < kMaxSites; ++s) {
      if (s < m) {
        const long long o = (long long)s * g.Nr + p;
        const double ts = t[o];
        gs[s] = closure_c<double>(closure, beta * v[o], ts) + ts + 1.0;
      }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int u = u0 + k;
      if (u >= n) break;
      const SiteP b = solute[u];
      const double ab[3] = {x - b.x, y - b.y, z - b.z};
      const double r = sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
      if (!(r > 0.0)) continue;
      double f = 0.0;
#pragma unroll
      for (int s = 0; s < kMaxSites; ++s) {
        if (s < m) {
          const SiteP a = solvent[s];
          const double eab = sqrt(a.epsilon * b.epsilon), sab = 0.5 * (a.sigma + b.sigma);
          const double qab = a.charge * b.charge * kEps0Inv;
          f += gs[s] * ((eab / sab) * ljcap1(r / sab) + qab * kG * kG * ccap1(kG * r));
        }
      }
      // drab = -ab[dim] / r
#pragma unroll
      for (int d = 0; d < 3; ++d) acc[k][d] -= f * (ab[d] / r);
    }
  }
  __shared__ double sm[U * 3][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < U; ++k)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double a = acc[k][d];
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0) sm[3 * k + d][wid] = a;
    }
  __syncthreads();
  if (threadIdx.x < U * 3) {
    const int u = u0 + threadIdx.x / 3;
    if (u < n) {
      double a = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sm[threadIdx.x][w];
      part[((long long)u * gridDim.x + blockIdx.x) * 3 + threadIdx.x % 3] = a;
    }
  }
}

// out = d + 1 (the closure's dh/dx, the slope the flagged Jacobian applies).
static __global__ void k_shift1(long long n, const double *__restrict__ d, double *__restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = d[i] + 1.0;
}

// Block partials of sum_r sum_s form1(x, dx, h, dh, c, dc, cl) with
// dx = -beta dv + dT, dc = c' dx - beta dv, dh = dc + dT (hnc3d.c:2063-2097).
static __global__ void __launch_bounds__(256) k_mu1(Geo g, const double *__restrict__ t,
                                                    const double *__restrict__ v, const double *__restrict__ uc,
                                                    const double *__restrict__ dv, const double *__restrict__ dT,
                                                    double beta, int closure, const double *__restrict__ charge,
                                                    double *__restrict__ part) {
  double acc = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.Nr;
       p += (long long)gridDim.x * blockDim.x) {
    for (int s = 0; s < g.m; ++s) {
      const long long o = (long long)s * g.Nr + p;
      const double ts = t[o], bv = beta * v[o];
      const double c = closure_c<double>(closure, bv, ts), d = closure_d<double>(closure, bv, ts);
      const double h = c + ts, x = -bv + ts, cl = -beta * charge[s] * uc[p];
      const double bdv = beta * dv[o], dt = dT[o];
      const double dx = -bdv + dt, dc = d * dx - bdv, dh = dc + dt;
      acc += form1(closure, x, dx, h, dh, c, dc, cl);
    }
  }
  __shared__ double sm[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) sm[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sm[w];
    part[blockIdx.x] = a;
  }
}

}  // namespace rism
