// solvent.cuh -- kernels of the 3D-RISM pure-solvent solve (hnc3d_solvent_solve,
// hnc3d.c:803-1073): the site-site residual iterate_t2 (hnc3d.c:353-456) and
// its Jacobian, run as the same five passes as the solute residual over the
// m(m+1)/2 pair fields t_ij (i >= j, pair p = i(i+1)/2 + j, the packing of
// vec_aliases_create2, bgy3d-vec.h:739-758).  Only the z pass differs: at
// every k it solves the molecular OZ equation
//
//   X = (1 - rho W C)^-1 W C W,   t = X - C
//
// for the m x m complex C(k) of all pairs at once (compute_t2_m,
// hnc3d.c:231-323, whose column-major zgemm / zgesv sequence reduces to this
// for symmetric W and C), with the intramolecular W(k) = sinc(k r_ij)
// (omega_intra, bgy3d-pure.c:241-276) and the long-range Coulomb
// -beta q_i q_j 4 pi/eps0 e^{-k^2/4G^2}/k^2 (bgy3d_pair_potential,
// bgy3d-force.c:123-147) evaluated on the fly.  The Jacobian (the reference
// has none and lets SNES difference F) differentiates A X = W C W:
// dX = A^-1 W dC (W + rho X), with C at the base point kept from the last
// residual evaluation.
#pragma once
#include "kernels.cuh"

namespace rism {

constexpr int kMaxSolventSites = 4;  // m; m(m+1)/2 <= 10 pair fields
enum { MODE_VL = 3 };                // z pass: the real-space long-range c_L = -beta v_L (no input)

template <int MS> struct PureParams {
  static constexpr int NP = MS * (MS + 1) / 2;
  double rho, beta, h3;
  double q2[NP];     // q_i q_j
  double wr[NP];     // 2 pi r_ij / L0 (omega_intra's k r = wr |n|)
  double2 *ck;       // [pair][N2][N1][Nhp]: C at the corner, written by MODE_F, read by MODE_J
};

// In-place LU with partial pivoting of a complex MS x MS matrix (rows
// swapped as recorded in piv) and the solve of A X = B for MS columns.
template <int MS> __device__ __forceinline__ void lu_factor(double2 (&A)[MS][MS], int (&piv)[MS]) {
#pragma unroll
  for (int k = 0; k < MS; ++k) {
    int p = k;
    double best = A[k][k].x * A[k][k].x + A[k][k].y * A[k][k].y;
#pragma unroll
    for (int i = k + 1; i < MS; ++i) {
      const double a = A[i][k].x * A[i][k].x + A[i][k].y * A[i][k].y;
      if (a > best) { best = a; p = i; }
    }
    piv[k] = p;
#pragma unroll
    for (int i = k + 1; i < MS; ++i)
      if (i == p)
#pragma unroll
        for (int j = 0; j < MS; ++j) { const double2 t = A[k][j]; A[k][j] = A[i][j]; A[i][j] = t; }
    const double2 d = A[k][k];
    const double dn = d.x * d.x + d.y * d.y;
#pragma unroll
    for (int i = k + 1; i < MS; ++i) {
      const double2 a = A[i][k];
      const double2 l = make_double2((a.x * d.x + a.y * d.y) / dn, (a.y * d.x - a.x * d.y) / dn);
      A[i][k] = l;
#pragma unroll
      for (int j = k + 1; j < MS; ++j) {
        A[i][j].x -= l.x * A[k][j].x - l.y * A[k][j].y;
        A[i][j].y -= l.x * A[k][j].y + l.y * A[k][j].x;
      }
    }
  }
}

template <int MS>
__device__ __forceinline__ void lu_solve(const double2 (&A)[MS][MS], const int (&piv)[MS], double2 (&B)[MS][MS]) {
#pragma unroll
  for (int k = 0; k < MS; ++k)
#pragma unroll
    for (int i = k + 1; i < MS; ++i)
      if (i == piv[k])
#pragma unroll
        for (int j = 0; j < MS; ++j) { const double2 t = B[k][j]; B[k][j] = B[i][j]; B[i][j] = t; }
#pragma unroll
  for (int j = 0; j < MS; ++j) {
#pragma unroll
    for (int i = 1; i < MS; ++i)
#pragma unroll
      for (int k = 0; k < i; ++k) {
        B[i][j].x -= A[i][k].x * B[k][j].x - A[i][k].y * B[k][j].y;
        B[i][j].y -= A[i][k].x * B[k][j].y + A[i][k].y * B[k][j].x;
      }
#pragma unroll
    for (int i = MS - 1; i >= 0; --i) {
      double2 s = B[i][j];
#pragma unroll
      for (int k = i + 1; k < MS; ++k) {
        s.x -= A[i][k].x * B[k][j].x - A[i][k].y * B[k][j].y;
        s.y -= A[i][k].x * B[k][j].y + A[i][k].y * B[k][j].x;
      }
      const double2 d = A[i][i];
      const double dn = d.x * d.x + d.y * d.y;
      B[i][j] = make_double2((s.x * d.x + s.y * d.y) / dn, (s.y * d.x - s.x * d.y) / dn);
    }
  }
}

__device__ __forceinline__ double sinc(double x) { return x == 0.0 ? 1.0 : sin(x) / x; }

// z pass of the pure solvent: forward z transform of the NP pair fields of a
// tile, the per-k OZ solve (MODE_F) or its differential (MODE_J), inverse z
// transform.  MODE_VL ignores the input and writes the long-range term
// -beta q2 v_L(k) / h^3 (centred) for the inverse transform.  Output in the
// units the x-inverse pass expects: t_centre(k) / h^3.
template <int MODE, int B, int MS>
__global__ void __launch_bounds__(256) k_z_oz(Geo g, AxisPlan pz, double2 *__restrict__ W, PureParams<MS> pp) {
  using V = double2;
  constexpr int NP = MS * (MS + 1) / 2;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + pz.n;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int kx0 = blockIdx.x * B;
  const int y = blockIdx.y;
  const int bw = min(B, g.Nh - kx0);
  const int N2 = g.N2;
  const V *twg = reinterpret_cast<const V *>(pz.tw);
  for (int q = tid; q < pz.n; q += nthr) tw[q] = twg[q];
  const long long zstride = (long long)g.N1 * g.Nhp;
  const long long col = (long long)y * g.Nhp + kx0;
  constexpr int mB = NP * B;
  if (MODE != MODE_VL) {
    for (int e = tid; e < N2 * mB; e += nthr) {
      const int z = e / mB, r = e - z * mB;
      const int s = r / B, b = r - s * B;
      V v = make_double2(0.0, 0.0);
      if (b < bw) v = W[(long long)s * g.Nc + z * zstride + col + b];
      buf[e] = v;
    }
    __syncthreads();
#pragma unroll 1
    for (int s = 0; s < NP; ++s) fft_tile<false, true>(buf + s * B, pz, B, mB, 1, tw);
  } else {
    __syncthreads();
  }
  const int ky = kfreq(y, g.N1);
  const double k1 = ky * g.dk1;
  const double h3 = pp.h3, rho = pp.rho, beta = pp.beta;
  for (int e = tid; e < N2 * B; e += nthr) {
    const int z = e / B, b = e - z * B;
    if (b >= bw) continue;
    const int kx = kx0 + b;
    const int kz = kfreq(z, N2);
    const double k0 = kx * g.dk0, k2 = kz * g.dk2;
    const double kk = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)), __dmul_rn(k2, k2)));
    const double kq = kk * kk;
    // coulomb_long_fourier(k, 1, G) (bgy3d-force.h:139-148)
    const double clf = kq == 0.0 ? 0.0 : (4 * M_PI * kEps0Inv) * exp(-kq / (4 * kG * kG)) / kq;
    const double sg = ((kx + ky + kz) & 1) ? -1.0 : 1.0;  // centre <-> corner
    const long long o = z * zstride + col + b;
    if (MODE == MODE_VL) {
#pragma unroll
      for (int p = 0; p < NP; ++p) buf[(z * NP + p) * B + b] = make_double2(-beta * pp.q2[p] * clf * sg / h3, 0.0);
      continue;
    }
    const double sqn = sqrt((double)(kx * kx + ky * ky + kz * kz));
    double Wm[MS][MS];
    V C[MS][MS], A[MS][MS], X[MS][MS], D[MS][MS];
#pragma unroll
    for (int i = 0; i < MS; ++i)
#pragma unroll
      for (int j = 0; j <= i; ++j) {
        const int p = i * (i + 1) / 2 + j;
        Wm[i][j] = Wm[j][i] = (i == j) ? 1.0 : sinc(pp.wr[p] * sqn);
        const V in = buf[(z * NP + p) * B + b];
        if (MODE == MODE_F) {
          // C = [FFT(c) h^3 - beta v_L] at the corner (hnc3d.c:382-405)
          const V cc = make_double2(in.x * h3 * sg - beta * pp.q2[p] * clf, in.y * h3 * sg);
          pp.ck[(long long)p * g.Nc + o] = cc;
          C[i][j] = C[j][i] = cc;
        } else {
          C[i][j] = C[j][i] = pp.ck[(long long)p * g.Nc + o];
          D[i][j] = D[j][i] = make_double2(in.x * h3 * sg, in.y * h3 * sg);  // dC
        }
      }
    // WC (into X), A = 1 - rho W C, R = (WC) W (into C's slot below)
#pragma unroll
    for (int i = 0; i < MS; ++i)
#pragma unroll
      for (int j = 0; j < MS; ++j) {
        V s = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < MS; ++k) { s.x += Wm[i][k] * C[k][j].x; s.y += Wm[i][k] * C[k][j].y; }
        X[i][j] = s;
        A[i][j] = make_double2((i == j ? 1.0 : 0.0) - rho * s.x, -rho * s.y);
      }
    V R[MS][MS];
#pragma unroll
    for (int i = 0; i < MS; ++i)
#pragma unroll
      for (int j = 0; j < MS; ++j) {
        V s = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < MS; ++k) { s.x += X[i][k].x * Wm[k][j]; s.y += X[i][k].y * Wm[k][j]; }
        R[i][j] = s;
      }
    int piv[MS];
    lu_factor<MS>(A, piv);
    lu_solve<MS>(A, piv, R);  // R <- X
    if (MODE == MODE_F) {
#pragma unroll
      for (int i = 0; i < MS; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
          const int p = i * (i + 1) / 2 + j;
          // back to the centre, long range out (hnc3d.c:411-437)
          const double tr = R[i][j].x - C[i][j].x - beta * pp.q2[p] * clf, ti = R[i][j].y - C[i][j].y;
          buf[(z * NP + p) * B + b] = make_double2(tr * sg / h3, ti * sg / h3);
        }
    } else {
      // Q = W + rho X (into X), Y = W dC Q (into A's row buffer via R2)
      V WD[MS][MS];
#pragma unroll
      for (int i = 0; i < MS; ++i)
#pragma unroll
        for (int j = 0; j < MS; ++j) {
          V s = make_double2(0.0, 0.0);
#pragma unroll
          for (int k = 0; k < MS; ++k) { s.x += Wm[i][k] * D[k][j].x; s.y += Wm[i][k] * D[k][j].y; }
          WD[i][j] = s;
          X[i][j] = make_double2(Wm[i][j] + rho * R[i][j].x, rho * R[i][j].y);
        }
#pragma unroll
      for (int i = 0; i < MS; ++i)
#pragma unroll
        for (int j = 0; j < MS; ++j) {
          V s = make_double2(0.0, 0.0);
#pragma unroll
          for (int k = 0; k < MS; ++k) {
            s.x += WD[i][k].x * X[k][j].x - WD[i][k].y * X[k][j].y;
            s.y += WD[i][k].x * X[k][j].y + WD[i][k].y * X[k][j].x;
          }
          R[i][j] = s;
        }
      lu_solve<MS>(A, piv, R);  // R <- dX
#pragma unroll
      for (int i = 0; i < MS; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
          const int p = i * (i + 1) / 2 + j;
          const double tr = R[i][j].x - D[i][j].x, ti = R[i][j].y - D[i][j].y;
          buf[(z * NP + p) * B + b] = make_double2(tr * sg / h3, ti * sg / h3);
        }
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int s = 0; s < NP; ++s) fft_tile<true, true>(buf + s * B, pz, B, mB, 1, tw);
  for (int e = tid; e < N2 * mB; e += nthr) {
    const int z = e / mB, r = e - z * mB;
    const int s = r / B, b = r - s * B;
    if (b < bw) W[(long long)s * g.Nc + z * zstride + col + b] = buf[e];
  }
}

// Site-site short-range potentials on the centred grid (bgy3d_pair_potential,
// bgy3d-force.c:123-147, lennard_jones_coulomb_short, bgy3d-force.h:30-98):
// LJ capped at eps * CUTOFF and the erfc(G r)/r Coulomb capped at CUTOFF2.
struct PairP { double sigma, epsilon, q2; };
constexpr double kCutoff = 1.0e8;            // bgy3d-force.h:10
constexpr double kCutoff2 = kCutoff * 1.0e-5;  // bgy3d-force.h:11

static __global__ void k_pair_field(Geo g, double h0, double h1, double h2, double L0, double L1, double L2,
                                    const PairP *__restrict__ pairs, double *__restrict__ v) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  const int i0 = (int)(p % g.N0);
  const int i1 = (int)((p / g.N0) % g.N1);
  const int i2 = (int)(p / ((long long)g.N0 * g.N1));
  const double x = i0 * h0 - L0 / 2, y = i1 * h1 - L1 / 2, z = i2 * h2 - L2 / 2;
  const double r = sqrt((x * x + y * y) + z * z);
  for (int s = 0; s < g.m; ++s) {
    const PairP a = pairs[s];
    double lj = 0.0;
    if (!((a.sigma == 0.0 || a.epsilon == 0.0) && r == 0.0)) {
      const double sr = a.sigma / r;
      const double sr6 = (sr * sr) * (sr * sr) * (sr * sr);
      const double re = 4 * a.epsilon * sr6 * (sr6 - 1);
      lj = (fabs(re) > a.epsilon * kCutoff) ? a.epsilon * kCutoff : re;
    }
    const double f = erfc(kG * r) / r;
    const double cs = f > kCutoff2 ? kEps0Inv * a.q2 * kCutoff2 : kEps0Inv * a.q2 * f;
    v[(long long)s * g.Nr + p] = lj + cs;
  }
}

// Radial tables (value, slope pairs on r = (i + 1/2) dr) onto the centred
// grid, one table per pair field (vec_rtab, bgy3d-vec.c:49-56).
static __global__ void k_rtab(Geo g, double h0, double h1, double h2, double L0, double L1, double L2,
                              const double2 *__restrict__ tab, int nrad, double dr, double *__restrict__ out) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  const int i0 = (int)(p % g.N0);
  const int i1 = (int)((p / g.N0) % g.N1);
  const int i2 = (int)(p / ((long long)g.N0 * g.N1));
  const double x = i0 * h0 - L0 / 2, y = i1 * h1 - L1 / 2, z = i2 * h2 - L2 / 2;
  const double r = sqrt((x * x + y * y) + z * z);
  const double ix = r / dr - 0.5;
  int i = (int)(ix + 0.5);
  i = min(max(i, 0), nrad - 1);
  const double fr = ix - i;
  for (int s = 0; s < g.m; ++s) {
    const double2 t = tab[(long long)s * nrad + i];
    out[(long long)s * g.Nr + p] = t.x + t.y * fr;
  }
}

// Block partials of the pure-solvent observables over all m x m pairs
// (off-diagonal pairs twice): the free-energy densities of the native
// closure, HNC, KH and GF (print_chempot, hnc3d.c:674-694) with
// x = -beta v + t, h = c + t and the FFT long-range cl (hnc3d.c:975-1008),
// and sum c (compute_kc, hnc3d.c:707-718); h written for the chi output and
// g = 1 + h when g is non-null.  part[block * 5 + {mu, hnc, kh, gf, c}].
static __global__ void __launch_bounds__(256) k_solvent_obs(Geo g, int ms, const double *__restrict__ t,
                                                            const double *__restrict__ v,
                                                            const double *__restrict__ cl, double beta, int closure,
                                                            double *__restrict__ h_out, double *__restrict__ g_out,
                                                            double *__restrict__ part) {
  double acc[5] = {0, 0, 0, 0, 0};
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.Nr;
       p += (long long)gridDim.x * blockDim.x) {
    int q = 0;
    for (int i = 0; i < ms; ++i)
      for (int j = 0; j <= i; ++j, ++q) {
        const long long o = (long long)q * g.Nr + p;
        const double ts = t[o], bv = beta * v[o];
        const double c = closure_c<double>(closure, bv, ts);
        const double h = c + ts, x = -bv + ts, l = cl[o];
        const double w = i == j ? 1.0 : 2.0;
        acc[0] += w * form(closure, x, h, c, l);
        acc[1] += w * form(CL_HNC, x, h, c, l);
        acc[2] += w * form(CL_KH, x, h, c, l);
        acc[3] += w * form(CL_PY, x, h, c, l);
        acc[4] += w * c;
        h_out[o] = h;
        if (g_out) g_out[o] = h + 1.0;
      }
  }
  __shared__ double sm[5][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double a = acc[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) sm[k][wid] = a;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sm[threadIdx.x][w];
    part[blockIdx.x * 5 + threadIdx.x] = a;
  }
}

// chi - 1 = rho FFT(h) h^3 at the corner, plus omega for i != j
// (hnc3d.c:1020-1043), from the forward transform of h in W into a dense
// [pair][N2][N1][N0/2+1] complex array.
template <int MS>
__global__ void k_chi_out(Geo g, const double2 *__restrict__ Wh, PureParams<MS> pp,
                          double2 *__restrict__ out) {
  const long long nk = (long long)g.Nh * g.N1 * g.N2;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nk; q += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(q % g.Nh);
    const int iy = (int)((q / g.Nh) % g.N1);
    const int iz = (int)(q / ((long long)g.Nh * g.N1));
    const int ky = kfreq(iy, g.N1), kz = kfreq(iz, g.N2);
    const double sg = ((kx + ky + kz) & 1) ? -1.0 : 1.0;
    const double sqn = sqrt((double)(kx * kx + ky * ky + kz * kz));
    const long long o = ((long long)iz * g.N1 + iy) * g.Nhp + kx;
#pragma unroll
    for (int i = 0; i < MS; ++i)
#pragma unroll
      for (int j = 0; j <= i; ++j) {
        const int p = i * (i + 1) / 2 + j;
        const double2 w = Wh[(long long)p * g.Nc + o];
        double2 r = make_double2(pp.rho * w.x * pp.h3 * sg, pp.rho * w.y * pp.h3 * sg);
        if (i != j) r.x += sinc(pp.wr[p] * sqn);
        out[(long long)p * nk + q] = r;
      }
  }
}

}  // namespace rism
