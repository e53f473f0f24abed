// kernels.cuh -- sm_100a kernels of the 3D-RISM solute residual and its
// Jacobian (hnc3d.c iterate_t1 / jacobian_t1), the setup fields and the
// Krylov vector operations.
//
// One residual evaluation F(t) = (chi-1)*c(t) - beta/eps0 tau - t for all m
// solvent sites is five passes over HBM:
//
//   k_xfwd  closure c(t) (or c'(t) dt) fused into the prologue of the
//           real-to-complex transform along x (half-length complex FFT +
//           untangling), writing the complex work buffer W;
//   k_y     complex transform along y, in place on W;
//   k_z     transform along z, the OZ contraction t_i = sum_j (chi-1)_ij c_j
//           against radial chi(|k|) tables, the renormalised long-range
//           term, and the inverse transform along z -- all on one tile in
//           shared memory, so the k-space product costs no extra HBM pass;
//   k_y     inverse along y;
//   k_xinv  complex-to-real along x, normalisation, "- t" and the residual
//           norms (warp-shuffle + per-block partials) in the epilogue.
//
// W is [m][N2][N1][Nhp] complex with Nhp >= N0/2+1 (kx fastest).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fft_core.cuh"

namespace rism {

constexpr int kMaxSites = 6;          // solvent sites m
constexpr double kEps0Inv = 331.84164;  // EPSILON0INV, bgy3d.h:145
constexpr double kG = 1.2;              // G_COULOMB_INVERSE_RANGE, bgy3d-solvents.h:9

// MODE_FWD: plain forward 3D transform of A (x and z passes; the z pass
// stops after its forward transform), used by the gradient.
enum { MODE_F = 0, MODE_J = 1, MODE_FWD = 2 };
enum { CL_HNC = 0, CL_KH = 1, CL_PY = 2, CL_PSE0 = 3 };

struct Geo {
  int N0, N1, N2;   // real grid
  int M;            // N0 / 2
  int Nh;           // N0 / 2 + 1
  int Nhp;          // padded complex row
  int m;            // solvent sites
  long long Nr;     // N0 * N1 * N2
  long long Nc;     // Nhp * N1 * N2
  double dk0, dk1, dk2;  // 2 pi / L
};

// ------------------------------------------------------------------ math
__device__ __forceinline__ double xexpm1(double x) { return expm1(x); }
__device__ __forceinline__ float xexpm1(float x) { return expm1f(x); }
__device__ __forceinline__ double xexp(double x) { return exp(x); }
__device__ __forceinline__ float xexp(float x) { return expf(x); }

// Truncated exponential series (closures.f90:191-236, Horner form).
template <typename T> __device__ __forceinline__ T exps1(int n, T x) {
  T c = T(1), y = T(0);
  for (int k = n; k >= 1; --k) { y = x * y + c; c = c * T(k); }
  return (x / c) * y;
}
template <typename T> __device__ __forceinline__ T pse(int n, T x) {
  return x < T(0) ? xexpm1(x) : exps1(n, x);
}

// c = closure(beta v, t) (closures.f90:107-128).  bv = beta * v.
template <typename T> __device__ __forceinline__ T closure_c(int method, T bv, T t) {
  const T x = -bv + t;
  switch (method) {
    case CL_HNC: return xexpm1(x) - t;
    case CL_KH: return x <= T(0) ? xexpm1(x) - t : -bv;
    case CL_PY: return xexp(-bv) * (T(1) + t) - T(1) - t;
    default: return pse(method - CL_PSE0, x) - t;
  }
}
// dc/dt (closures.f90:131-153): closure1 == closure_d * dt.
template <typename T> __device__ __forceinline__ T closure_d(int method, T bv, T t) {
  const T x = -bv + t;
  switch (method) {
    case CL_HNC: return xexpm1(x);
    case CL_KH: return x <= T(0) ? xexpm1(x) : T(0);
    default: return pse(method - CL_PSE0 - 1, x);
  }
}

__device__ __forceinline__ double dfact(int n) {
  double f = 1.0;
  for (int k = 2; k <= n; ++k) f *= k;
  return f;
}
// beta mu / rho density (closures.f90:574-612).
__device__ __forceinline__ double form(int method, double x, double h, double c, double cl) {
  const double base = -c - h * (c + cl) / 2;
  switch (method) {
    case CL_HNC: return base + h * h / 2;
    case CL_KH: return h < 0 ? base + h * h / 2 : base;
    case CL_PY: return base;
    default: {
      if (h < 0) return base + h * h / 2;
      const int mm = method - CL_PSE0 + 1;
      double xm = 1.0;
      for (int k = 0; k < mm; ++k) xm *= x;
      return base + (h * h / 2 - xm / dfact(mm));
    }
  }
}

__device__ __forceinline__ int kfreq(int i, int n) { return i <= n / 2 ? i : i - n; }

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// ------------------------------------------------------------- reductions
struct NormPartial { double amax, sum2; };

// out[0] = the largest amax (a NaN anywhere gives NaN), out[1] = the sum of
// sum2, out[2] = *err: the block partials of one residual reduced on the
// device in one fixed order (strided per thread, then a pairwise tree), so
// that three doubles, not the partials, cross to the host.
__device__ __forceinline__ double amax_merge(double a, double x) { return (a != a) ? a : ((x > a || x != x) ? x : a); }
__global__ static void __launch_bounds__(1024) k_norm_final(int nblk, const NormPartial *__restrict__ part,
                                                            const int *__restrict__ err, double *__restrict__ out) {
  __shared__ double sa[1024], ss[1024];
  const int t = threadIdx.x;
  double a = 0.0, s = 0.0;
  for (int b = t; b < nblk; b += 1024) {
    a = amax_merge(a, part[b].amax);
    s += part[b].sum2;
  }
  sa[t] = a;
  ss[t] = s;
  __syncthreads();
  for (int st = 512; st > 0; st >>= 1) {
    if (t < st) {
      sa[t] = amax_merge(sa[t], sa[t + st]);
      ss[t] += ss[t + st];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = sa[0];
    out[1] = ss[0];
    out[2] = (double)*err;
  }
}

__device__ __forceinline__ void block_norms(double amax, double sum2, NormPartial *out) {
  for (int o = 16; o > 0; o >>= 1) {
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    sum2 += __shfl_xor_sync(0xffffffffu, sum2, o);
  }
  __shared__ double s_a[32], s_s[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { s_a[wid] = amax; s_s[wid] = sum2; }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    amax = lane < nw ? s_a[lane] : 0.0;
    sum2 = lane < nw ? s_s[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
      sum2 += __shfl_xor_sync(0xffffffffu, sum2, o);
    }
    if (lane == 0) out->amax = amax, out->sum2 = sum2;
  }
}

// ============================================================ FFT passes
// x forward: closure (MODE_F: A = t, B = v, p = beta) or linearised closure
// (MODE_J: A = dt, B = d = dc/dt, p = scale of dt) fused into the r2c
// transform of RX rows of N0 reals.
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_xfwd(Geo g, AxisPlan px, int RX, const T *__restrict__ A,
                                             const T *__restrict__ B, T p, int closure,
                                             typename Cx<T>::type *__restrict__ W,
                                             const typename Cx<T>::type *__restrict__ post) {
  using V = typename Cx<T>::type;
  using P2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + px.n;
  const int M = g.M;
  const int rows_total = g.N1 * g.N2;
  const int row0 = blockIdx.x * RX;
  const int site = blockIdx.y;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const V *twg = reinterpret_cast<const V *>(px.tw);
  for (int q = tid; q < px.n; q += nthr) tw[q] = twg[q];
  const long long sbase = (long long)site * g.Nr;
  for (int e = tid; e < RX * M; e += nthr) {
    const int row = e / M, j = e - row * M;
    const int grow = row0 + row;
    V z;
    z.x = T(0); z.y = T(0);
    if (grow < rows_total) {
      const long long off = sbase + (long long)grow * g.N0 + 2 * j;
      const P2 a = *reinterpret_cast<const P2 *>(A + off);
      const P2 b = *reinterpret_cast<const P2 *>(B + off);
      if (MODE == MODE_F) {
        z.x = closure_c<T>(closure, p * b.x, a.x);
        z.y = closure_c<T>(closure, p * b.y, a.y);
      } else if (MODE == MODE_FWD) {
        z.x = a.x * p;
        z.y = a.y * p;
      } else {
        z.x = b.x * (a.x * p);
        z.y = b.y * (a.y * p);
      }
    }
    buf[e] = z;
  }
  __syncthreads();
  fft_tile<false, false>(buf, px, RX, 1, M, tw);
  const int H = M / 2 + 1;
  const long long wbase = (long long)site * g.Nc;
  for (int e = tid; e < RX * H; e += nthr) {
    const int row = e / H, k = e - row * H;
    const int grow = row0 + row;
    if (grow >= rows_total) continue;
    const V zk = buf[row * M + (k == 0 ? 0 : k)];
    const V zm = buf[row * M + (k == 0 ? 0 : M - k)];
    // E = (Zk + conj Zm)/2, O = (Zk - conj Zm)/(2i); X_k = E + w O, X_{M-k} = conj(E - w O)
    V E, O;
    E.x = (zk.x + zm.x) * T(0.5);
    E.y = (zk.y - zm.y) * T(0.5);
    O.x = (zk.y + zm.y) * T(0.5);
    O.y = -(zk.x - zm.x) * T(0.5);
    const V wO = cmul(post[k], O);
    V *row_out = W + wbase + (long long)grow * g.Nhp;
    row_out[k] = cadd(E, wO);
    if (M - k != k) row_out[M - k] = cconj(csub(E, wO));
  }
}

// y pass (forward or inverse), in place on W, tile of B kx-columns.
template <typename T, bool INV, int B>
__global__ void __launch_bounds__(256) k_y(Geo g, AxisPlan py, typename Cx<T>::type *__restrict__ W) {
  using V = typename Cx<T>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + py.n;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int kx0 = blockIdx.x * B;
  const int z = blockIdx.y, site = blockIdx.z;
  const int bw = min(B, g.Nh - kx0);
  const V *twg = reinterpret_cast<const V *>(py.tw);
  for (int q = tid; q < py.n; q += nthr) tw[q] = twg[q];
  V *base = W + (long long)site * g.Nc + (long long)z * g.N1 * g.Nhp + kx0;
  const int N1 = g.N1;
  for (int e = tid; e < N1 * B; e += nthr) {
    const int y = e / B, b = e - y * B;
    V v;
    v.x = T(0); v.y = T(0);
    if (b < bw) v = base[(long long)y * g.Nhp + b];
    buf[e] = v;
  }
  __syncthreads();
  fft_tile<INV, true>(buf, py, B, B, 1, tw);
  for (int e = tid; e < N1 * B; e += nthr) {
    const int y = e / B, b = e - y * B;
    if (b < bw) base[(long long)y * g.Nhp + b] = buf[e];
  }
}

// Parameters of the k-space step (hnc3d.c:1208-1262).
template <typename T> struct ZParams {
  const typename Vec2<T>::type *chi;   // [m(m+1)/2][nrad] (value, slope) of chi-1
  const typename Vec2<T>::type *stab;  // [m][nrad] (value, slope) of beta/eps0 s_i, or null
  const typename Cx<T>::type *L;       // [N2][N1][Nhp] long-range field / h^3, or null
  const typename Cx<T>::type *chi3;    // chi - 1 on the k grid [m(m+1)/2][N2][N1][Nhp], or null
  int nrad;
  double dkr;                          // pi / rmax
  T a[kMaxSites];                      // c_j -= a_j L      (no-renorm: beta q_j)
  T bconst[kMaxSites];                 // t_i -= bconst_i L (no-renorm: beta q_i)
};

// z pass: forward transform along z of all m sites, OZ contraction with the
// radial chi-1 tables (+ long-range terms in MODE_F), inverse along z.
template <typename T, int MODE, int B>
__global__ void __launch_bounds__(256) k_z(Geo g, AxisPlan pz, typename Cx<T>::type *__restrict__ W,
                                          ZParams<T> zp) {
  using V = typename Cx<T>::type;
  using P2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + pz.n;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int m = g.m;
  const int kx0 = blockIdx.x * B;
  const int y = blockIdx.y;
  const int bw = min(B, g.Nh - kx0);
  const int N2 = g.N2;
  const V *twg = reinterpret_cast<const V *>(pz.tw);
  for (int q = tid; q < pz.n; q += nthr) tw[q] = twg[q];
  const long long zstride = (long long)g.N1 * g.Nhp;
  const long long col = (long long)y * g.Nhp + kx0;
  const int mB = m * B;
  for (int e = tid; e < N2 * mB; e += nthr) {
    const int z = e / mB, r = e - z * mB;
    const int s = r / B, b = r - s * B;
    V v;
    v.x = T(0); v.y = T(0);
    if (b < bw) v = W[(long long)s * g.Nc + z * zstride + col + b];
    buf[e] = v;
  }
  __syncthreads();
  for (int s = 0; s < m; ++s) fft_tile<false, true>(buf + s * B, pz, B, mB, 1, tw);
  if (MODE == MODE_FWD) {
    __syncthreads();
    for (int e = tid; e < N2 * mB; e += nthr) {
      const int z = e / mB, r = e - z * mB;
      const int s = r / B, b = r - s * B;
      if (b < bw) W[(long long)s * g.Nc + z * zstride + col + b] = buf[e];
    }
    return;
  }
  const int ky = kfreq(y, g.N1);
  const double k1 = ky * g.dk1;
  for (int e = tid; e < N2 * B; e += nthr) {
    const int z = e / B, b = e - z * B;
    if (b >= bw) continue;
    const int kx = kx0 + b;
    const int kz = kfreq(z, N2);
    const double k0 = kx * g.dk0, k2 = kz * g.dk2;
    const double kk = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)), __dmul_rn(k2, k2)));
    int i = 0;
    T fr = T(0);
    if (zp.chi3 == nullptr) {
      const double ix = kk / zp.dkr - 0.5;
      i = (int)(ix + 0.5);
      i = min(max(i, 0), zp.nrad - 1);
      fr = T(ix - i);
    }
    V c[kMaxSites];
#pragma unroll
    for (int j = 0; j < kMaxSites; ++j)
      if (j < m) c[j] = buf[(z * m + j) * B + b];
    V Lk;
    Lk.x = T(0); Lk.y = T(0);
    if (MODE == MODE_F && zp.L != nullptr) {
      Lk = zp.L[z * zstride + col + b];
#pragma unroll
      for (int j = 0; j < kMaxSites; ++j)
        if (j < m) { c[j].x -= zp.a[j] * Lk.x; c[j].y -= zp.a[j] * Lk.y; }
    }
#pragma unroll
    for (int ii = 0; ii < kMaxSites; ++ii) {
      if (ii >= m) break;
      V t;
      t.x = T(0); t.y = T(0);
#pragma unroll
      for (int j = 0; j < kMaxSites; ++j) {
        if (j >= m) break;
        const int pidx = ii >= j ? ii * (ii + 1) / 2 + j : j * (j + 1) / 2 + ii;
        if (zp.chi3 != nullptr) {  // complex chi - 1 of the 3D solvent
          const V x = zp.chi3[(long long)pidx * g.Nc + z * zstride + col + b];
          t.x += x.x * c[j].x - x.y * c[j].y;
          t.y += x.x * c[j].y + x.y * c[j].x;
        } else {
          const P2 tv = zp.chi[(long long)pidx * zp.nrad + i];
          const T x = tv.x + tv.y * fr;
          t.x += x * c[j].x;
          t.y += x * c[j].y;
        }
      }
      if (MODE == MODE_F && zp.L != nullptr) {
        T bb = zp.bconst[ii];
        if (zp.stab != nullptr) {
          const P2 sv = zp.stab[(long long)ii * zp.nrad + i];
          bb += sv.x + sv.y * fr;
        }
        t.x -= bb * Lk.x;
        t.y -= bb * Lk.y;
      }
      buf[(z * m + ii) * B + b] = t;
    }
  }
  __syncthreads();
  for (int s = 0; s < m; ++s) fft_tile<true, true>(buf + s * B, pz, B, mB, 1, tw);
  for (int e = tid; e < N2 * mB; e += nthr) {
    const int z = e / mB, r = e - z * mB;
    const int s = r / B, b = r - s * B;
    if (b < bw) W[(long long)s * g.Nc + z * zstride + col + b] = buf[e];
  }
}

// x inverse: complex-to-real of RX rows, out = scale * x - sub * In, and the
// per-block residual norms of out.
template <typename T>
__global__ void __launch_bounds__(256) k_xinv(Geo g, AxisPlan px, int RX,
                                             const typename Cx<T>::type *__restrict__ W,
                                             const T *__restrict__ In, T *__restrict__ Out, T scale,
                                             T sub, const typename Cx<T>::type *__restrict__ post,
                                             NormPartial *__restrict__ part) {
  using V = typename Cx<T>::type;
  using P2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + px.n;
  const int M = g.M;
  const int rows_total = g.N1 * g.N2;
  const int row0 = blockIdx.x * RX;
  const int site = blockIdx.y;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const V *twg = reinterpret_cast<const V *>(px.tw);
  for (int q = tid; q < px.n; q += nthr) tw[q] = twg[q];
  const int H = M / 2 + 1;
  const long long wbase = (long long)site * g.Nc;
  for (int e = tid; e < RX * H; e += nthr) {
    const int row = e / H, k = e - row * H;
    const int grow = row0 + row;
    V zk, zm;
    zk.x = zk.y = zm.x = zm.y = T(0);
    if (grow < rows_total) {
      const V *row_in = W + wbase + (long long)grow * g.Nhp;
      V xk = row_in[k];
      V xm = row_in[M - k];
      // The 1D c2r stage reads only the real parts of the kx = 0 and
      // kx = N0/2 elements (as FFTW / pocketfft do).  They are real for a
      // Hermitian spectrum; the long-range term is not Hermitian on the ky /
      // kz Nyquist planes, which leaves imaginary parts here.
      if (k == 0) { xk.y = T(0); xm.y = T(0); }
      // A = X_k + conj X_{M-k}, D = X_k - conj X_{M-k}, P = D conj(w_k)
      V Aa, D;
      Aa.x = xk.x + xm.x; Aa.y = xk.y - xm.y;
      D.x = xk.x - xm.x;  D.y = xk.y + xm.y;
      const V Pp = cmul(D, cconj(post[k]));
      // Z_k = A + i P, Z_{M-k} = conj(A - i P)
      zk.x = Aa.x - Pp.y; zk.y = Aa.y + Pp.x;
      zm.x = Aa.x + Pp.y; zm.y = -(Aa.y - Pp.x);
    }
    buf[row * M + k] = zk;
    if (k != 0 && M - k != k) buf[row * M + (M - k)] = zm;
  }
  __syncthreads();
  fft_tile<true, false>(buf, px, RX, 1, M, tw);
  double amax = 0.0, sum2 = 0.0;
  const long long sbase = (long long)site * g.Nr;
  for (int e = tid; e < RX * M; e += nthr) {
    const int row = e / M, j = e - row * M;
    const int grow = row0 + row;
    if (grow >= rows_total) continue;
    const long long off = sbase + (long long)grow * g.N0 + 2 * j;
    const V z = buf[e];
    const P2 in = *reinterpret_cast<const P2 *>(In + off);
    P2 o;
    o.x = z.x * scale - sub * in.x;
    o.y = z.y * scale - sub * in.y;
    *reinterpret_cast<P2 *>(Out + off) = o;
    const double ox = (double)o.x, oy = (double)o.y;
    amax = fmax(amax, fmax(fabs(ox), fabs(oy)));
    sum2 += ox * ox + oy * oy;
  }
  block_norms(amax, sum2, part + (blockIdx.y * gridDim.x + blockIdx.x));
}

// ============================================================ setup fields
struct SiteP { double x, y, z, sigma, epsilon, charge; };

// r^-6 as (1/r^2)^3: one division instead of a general pow (a few ulp apart)
__device__ __forceinline__ double inv_pow6(double r) {
  const double i2 = 1.0 / (r * r);
  return i2 * i2 * i2;
}
__device__ __forceinline__ double lj0(double r) { const double p6 = inv_pow6(r); return 4 * p6 * (p6 - 1); }
__device__ __forceinline__ double lj1(double r) { const double p6 = inv_pow6(r); return 4 * p6 * (6 - 12 * p6) / r; }
__device__ __forceinline__ double ljcap0(double r) {   // bgy3d-solutes.c:101-114
  const double R = 0.2;
  if (r >= R) return lj0(r);
  const double b = lj1(R) / (2 * R), a = lj0(R);
  return a + b * (r - R) * (r + R);
}
__device__ __forceinline__ double cs0(double r) { return erfc(r) / r; }
__device__ __forceinline__ double cs1(double r) {
  const double r2 = r * r;
  return -(erfc(r) + (2 / sqrt(M_PI)) * r * exp(-r2)) / r2;
}
__device__ __forceinline__ double cscap0(double r) {  // bgy3d-solutes.c:230-243
  const double R = 0.2;
  if (r >= R) return cs0(r);
  const double b = cs1(R) / (2 * R), a = cs0(R);
  return a + b * (r - R) * (r + R);
}
__device__ __forceinline__ double cl0(double r) {     // bgy3d-solutes.c:147-159
  if (r >= 0.02) return erf(r) / r;
  const double r2 = r * r;
  return (2 / sqrt(M_PI)) * (1. + r2 * (-1. / 3. + r2 * (1. / 10. + r2 * (-1. / 42.))));
}

// v[i][p] = sum_u eps_iu ljcap0(r/sigma_iu) + q_i q_u/eps0 G cscap0(G r)
// (field0, bgy3d-solutes.c:343-377); grid point r = i h - L/2.  The pair
// constants (eps_iu, 1/sigma_iu, sigma_iu^2, q_i q_u / eps0) and the solute
// positions sit in shared memory ([n][m][4] then [n][3] doubles,
// kField0MaxPairs pairs and 384 sites at most).  Per point and solute site
// one 1/r^2 and one capped Coulomb value serve all solvent sites; per pair
// r/sigma is a product and (sigma/r)^6 = (sigma^2 / r^2)^3 (a few ulp from
// the division form below).  The terms sum in the same order.
constexpr int kField0MaxPairs = 1152;
static __global__ void __launch_bounds__(256) k_field0_pairs(Geo g, double h0, double h1, double h2, double L0,
                                                             double L1, double L2, const SiteP *__restrict__ solvent,
                                                             int n, const SiteP *__restrict__ solute,
                                                             double *__restrict__ v) {
  extern __shared__ double sp[];
  const int m = g.m;
  double *sx = sp + 4 * n * m;
  for (int e = threadIdx.x; e < n * m; e += blockDim.x) {
    const int u = e / m, s = e - u * m;
    const SiteP a = solvent[s], b = solute[u];
    const double sab = 0.5 * (a.sigma + b.sigma);
    sp[4 * e] = sqrt(a.epsilon * b.epsilon);
    sp[4 * e + 1] = 1.0 / sab;
    sp[4 * e + 2] = sab * sab;
    sp[4 * e + 3] = a.charge * b.charge * kEps0Inv;
  }
  for (int u = threadIdx.x; u < n; u += blockDim.x) {
    sx[3 * u] = solute[u].x;
    sx[3 * u + 1] = solute[u].y;
    sx[3 * u + 2] = solute[u].z;
  }
  __syncthreads();
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  const int i0 = (int)(p % g.N0);
  const int i1 = (int)((p / g.N0) % g.N1);
  const int i2 = (int)(p / ((long long)g.N0 * g.N1));
  const double x = i0 * h0 - L0 / 2, y = i1 * h1 - L1 / 2, z = i2 * h2 - L2 / 2;
  double e[kMaxSites];
#pragma unroll
  for (int s = 0; s < kMaxSites; ++s) e[s] = 0.0;
  for (int u = 0; u < n; ++u) {
    const double dx = x - sx[3 * u], dy = y - sx[3 * u + 1], dz = z - sx[3 * u + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double rab = sqrt(r2);
    const double cs = cscap0(kG * rab);
    const double ir2 = 1.0 / r2;  // inf on a site, where every pair takes the capped branch
    const double *c = sp + 4 * u * m;
#pragma unroll
    for (int s = 0; s < kMaxSites; ++s) {
      if (s < m) {
        const double xr = rab * c[4 * s + 1];
        double lj;
        if (xr >= 0.2) {  // ljcap0's cap radius
          const double i2 = c[4 * s + 2] * ir2, p6 = i2 * i2 * i2;
          lj = 4 * p6 * (p6 - 1);
        } else {
          lj = ljcap0(xr);
        }
        e[s] += c[4 * s] * lj + c[4 * s + 3] * kG * cs;
      }
    }
  }
#pragma unroll
  for (int s = 0; s < kMaxSites; ++s)
    if (s < m) v[(long long)s * g.Nr + p] = e[s];
}

static __global__ void k_field0(Geo g, double h0, double h1, double h2, double L0, double L1, double L2,
                         const SiteP *__restrict__ solvent, int n, const SiteP *__restrict__ solute,
                         double *__restrict__ v) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  const int i0 = (int)(p % g.N0);
  const int i1 = (int)((p / g.N0) % g.N1);
  const int i2 = (int)(p / ((long long)g.N0 * g.N1));
  const double x = i0 * h0 - L0 / 2, y = i1 * h1 - L1 / 2, z = i2 * h2 - L2 / 2;
  for (int s = 0; s < g.m; ++s) {
    const SiteP a = solvent[s];
    double e = 0.0;
    for (int u = 0; u < n; ++u) {
      const SiteP b = solute[u];
      const double eab = sqrt(a.epsilon * b.epsilon);
      const double sab = 0.5 * (a.sigma + b.sigma);
      const double qab = a.charge * b.charge * kEps0Inv;
      const double dx = x - b.x, dy = y - b.y, dz = z - b.z;
      const double rab = sqrt(dx * dx + dy * dy + dz * dz);
      e += eab * ljcap0(rab / sab) + qab * kG * cscap0(kG * rab);
    }
    v[(long long)s * g.Nr + p] = e;
  }
}

// uc(r) = (1/eps0) sum_u q_u G cl0(G r) (coulomb_long, bgy3d-solutes.c:795-815).
static __global__ void k_coulomb_long(Geo g, double h0, double h1, double h2, double L0, double L1, double L2,
                               int n, const SiteP *__restrict__ solute, double *__restrict__ uc) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.Nr) return;
  const int i0 = (int)(p % g.N0);
  const int i1 = (int)((p / g.N0) % g.N1);
  const int i2 = (int)(p / ((long long)g.N0 * g.N1));
  const double x = i0 * h0 - L0 / 2, y = i1 * h1 - L1 / 2, z = i2 * h2 - L2 / 2;
  double s = 0.0;
  for (int u = 0; u < n; ++u) {
    const double dx = x - solute[u].x, dy = y - solute[u].y, dz = z - solute[u].z;
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    s += solute[u].charge * kG * cl0(kG * r);
  }
  uc[p] = kEps0Inv * s;
}

// Per-axis phase factors of the solute form factor: tab[u][i] = exp(-i k_a(i)
// x_{u,a}) for axis a, i < n_a (k_a(i) = kfreq(i, Nfull_a) dk_a); so that
// exp(-i k.x_u) = tab0[u][ix] tab1[u][iy] tab2[u][iz].
static __global__ void k_phase_axis(int n, int na, int nfull, double dk, int axis, const SiteP *__restrict__ solute,
                                    double2 *__restrict__ tab) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * na) return;
  const int u = e / na, i = e - u * na;
  const double xu = axis == 0 ? solute[u].x : (axis == 1 ? solute[u].y : solute[u].z);
  double sn, cs;
  sincos(kfreq(i, nfull) * dk * xu, &sn, &cs);
  tab[e] = make_double2(cs, -sn);
}

// Long-range k-field, centred (bgy3d_solute_form, bgy3d-solutes.c:633-698):
// F(k) = sum_u q_u exp(-i k.x_u) (-1)^(kx+ky+kz).  renorm: L = F / h^3;
// no-renorm: L = (4 pi/eps0) exp(-k^2/4G^2)/k^2 F / h^3 (coulomb_long_fft,
// bgy3d-solutes.c:766-792; zero at k = 0).  Written in FP64 and FP32.  The
// phase of site u is the product of its three per-axis factors (k_phase_axis).
static __global__ void k_longrange_tab(Geo g, int n, const SiteP *__restrict__ solute,
                                       const double2 *__restrict__ t0, const double2 *__restrict__ t1,
                                       const double2 *__restrict__ t2, int renorm, double inv_h3,
                                       double2 *__restrict__ L64, float2 *__restrict__ L32) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long tot = (long long)g.Nh * g.N1 * g.N2;
  if (p >= tot) return;
  const int ix = (int)(p % g.Nh);
  const int iy = (int)((p / g.Nh) % g.N1);
  const int iz = (int)(p / ((long long)g.Nh * g.N1));
  const int fx = kfreq(ix, g.N0), fy = kfreq(iy, g.N1), fz = kfreq(iz, g.N2);
  double re = 0.0, im = 0.0;
  for (int u = 0; u < n; ++u) {
    const double2 a = t0[(long long)u * g.Nh + ix], b = t1[(long long)u * g.N1 + iy], c = t2[(long long)u * g.N2 + iz];
    const double br = a.x * b.x - a.y * b.y, bi = a.x * b.y + a.y * b.x;
    const double q = solute[u].charge;
    re += q * (br * c.x - bi * c.y);
    im += q * (br * c.y + bi * c.x);
  }
  const int sgn = (((fx % 2) != 0) ^ ((fy % 2) != 0) ^ ((fz % 2) != 0)) ? -1 : 1;
  double f = sgn * inv_h3;
  if (!renorm) {
    const double k0 = fx * g.dk0, k1 = fy * g.dk1, k2 = fz * g.dk2;
    const double kk = (k0 * k0 + k1 * k1) + k2 * k2;
    f *= kk == 0.0 ? 0.0 : (4 * M_PI * kEps0Inv) * exp(-kk / (4 * kG * kG)) / kk;
  }
  const long long o = ((long long)iz * g.N1 + iy) * g.Nhp + ix;
  L64[o] = make_double2(re * f, im * f);
  L32[o] = make_float2((float)(re * f), (float)(im * f));
}

// d_i = dc/dt at (v_i, t_i), in the precision of the Jacobian passes.
template <typename TO>
__global__ void k_closure_slope(long long n, long long Nr, const double *__restrict__ t,
                                const double *__restrict__ v, double beta, int closure, TO *__restrict__ d) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  d[p] = (TO)closure_d<double>(closure, beta * v[p], t[p]);
}

// Post-processing partials (hnc3d.c:2157-2269): per block sums of the mu
// densities by the native, HNC, KH and GF functionals and of c; g = h + 1.
struct ObsPartial { double mu, hnc, kh, gf, csum; };

// out[0..4] = the sums of the five fields of part[0..nblk): one block of
// 1024 threads, strided per thread, then a pairwise tree (a fixed order).
__global__ static void __launch_bounds__(1024) k_obs_final(int nblk, const ObsPartial *__restrict__ part,
                                                           double *__restrict__ out) {
  __shared__ double red[5][1024];
  const int t = threadIdx.x;
  double a[5] = {0, 0, 0, 0, 0};
  for (int b = t; b < nblk; b += 1024) {
    const ObsPartial p = part[b];
    a[0] += p.mu; a[1] += p.hnc; a[2] += p.kh; a[3] += p.gf; a[4] += p.csum;
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) red[q][t] = a[q];
  __syncthreads();
  for (int st = 512; st > 0; st >>= 1) {
    if (t < st) {
#pragma unroll
      for (int q = 0; q < 5; ++q) red[q][t] += red[q][t + st];
    }
    __syncthreads();
  }
  if (t < 5) out[t] = red[t][0];
}

static __global__ void k_observables(Geo g, const double *__restrict__ t, const double *__restrict__ v,
                              const double *__restrict__ uc, double beta, int closure,
                              const double *__restrict__ charge, double *__restrict__ gout,
                              ObsPartial *__restrict__ part) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double a[5] = {0, 0, 0, 0, 0};
  if (p < g.Nr) {
    for (int s = 0; s < g.m; ++s) {
      const long long o = (long long)s * g.Nr + p;
      const double ts = t[o], vs = v[o];
      const double c = closure_c<double>(closure, beta * vs, ts);
      const double h = c + ts;
      const double x = -beta * vs + ts;
      const double cl = 0.0 + (-beta * charge[s]) * uc[p];
      a[0] += form(closure, x, h, c, cl);
      a[1] += form(CL_HNC, x, h, c, cl);
      a[2] += form(CL_KH, x, h, c, cl);
      a[3] += form(CL_PY, x, h, c, cl);
      a[4] += c;
      if (gout) gout[o] = h + 1.0;
    }
  }
  for (int k = 0; k < 5; ++k)
    for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
  __shared__ double s[5][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 5; ++k) s[k][wid] = a[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double b[5] = {0, 0, 0, 0, 0};
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w)
      for (int k = 0; k < 5; ++k) b[k] += s[k][w];
    part[blockIdx.x] = ObsPartial{b[0], b[1], b[2], b[3], b[4]};
  }
}

// ============================================================ vector ops
// Krylov basis vectors are (pointer, scale) pairs so normalisation never
// needs its own pass.
template <typename T> struct VecRef { const T *p; double s; };
constexpr int kDotChunk = 8;

// partial[b][v] = sum over the block's range of w * (s_v V_v).
template <typename T>
__global__ void __launch_bounds__(256) k_mdot(long long n, const T *__restrict__ w, double ws, int nv,
                                             VecRef<T> v0, VecRef<T> v1, VecRef<T> v2, VecRef<T> v3,
                                             VecRef<T> v4, VecRef<T> v5, VecRef<T> v6, VecRef<T> v7,
                                             double *__restrict__ part) {
  const VecRef<T> vs[kDotChunk] = {v0, v1, v2, v3, v4, v5, v6, v7};
  double acc[kDotChunk];
#pragma unroll
  for (int k = 0; k < kDotChunk; ++k) acc[k] = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double wi = (double)w[i];
#pragma unroll
    for (int k = 0; k < kDotChunk; ++k)
      if (k < nv) acc[k] += wi * (double)vs[k].p[i];
  }
  __shared__ double s[kDotChunk][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kDotChunk; ++k) {
    double a = acc[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) s[k][wid] = a;
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double a = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a += s[threadIdx.x][q];
    part[(long long)blockIdx.x * kDotChunk + threadIdx.x] = a * ws * vs[threadIdx.x].s;
  }
}

// w = ws * w - sum_v c_v (s_v V_v); optional per-block sum of squares of w.
template <typename T>
__global__ void __launch_bounds__(256) k_maxpy(long long n, T *__restrict__ w, double ws, int nv,
                                              VecRef<T> v0, VecRef<T> v1, VecRef<T> v2, VecRef<T> v3,
                                              VecRef<T> v4, VecRef<T> v5, VecRef<T> v6, VecRef<T> v7,
                                              const double *__restrict__ coef, double *__restrict__ part) {
  const VecRef<T> vs[kDotChunk] = {v0, v1, v2, v3, v4, v5, v6, v7};
  double cf[kDotChunk];
#pragma unroll
  for (int k = 0; k < kDotChunk; ++k) cf[k] = k < nv ? coef[k] * vs[k].s : 0.0;
  double sum2 = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double a = ws == 0.0 ? 0.0 : ws * (double)w[i];
#pragma unroll
    for (int k = 0; k < kDotChunk; ++k)
      if (k < nv) a -= cf[k] * (double)vs[k].p[i];
    const T r = (T)a;
    w[i] = r;
    sum2 += (double)r * (double)r;
  }
  if (part) {
    for (int o = 16; o > 0; o >>= 1) sum2 += __shfl_xor_sync(0xffffffffu, sum2, o);
    __shared__ double s[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s[wid] = sum2;
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a += s[q];
      part[blockIdx.x] = a;
    }
  }
}

// y = a * x + b * y with arbitrary input/output precisions.
template <typename TX, typename TY>
__global__ void k_axpby(long long n, double a, const TX *__restrict__ x, double b, TY *__restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double yi = b == 0.0 ? 0.0 : b * (double)y[i];
    y[i] = (TY)(a * (double)x[i] + yi);
  }
}

// z = x + a * y (z may alias x), any precisions.
template <typename TX, typename TY, typename TZ>
__global__ void k_xpay(long long n, const TX *__restrict__ x, double a, const TY *__restrict__ y,
                       TZ *__restrict__ z) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    z[i] = (TZ)((double)x[i] + a * (double)y[i]);
}

}  // namespace rism
