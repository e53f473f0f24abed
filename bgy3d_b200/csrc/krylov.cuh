// krylov.cuh -- Gram-Schmidt kernels of the GMRES driver.
//
// Classical Gram-Schmidt needs two passes per Krylov step: h = V^T w (all
// previous basis vectors against the new one) and w -= V h (with ||w||).
// Both read the new vector once and up to kVecMax basis vectors in the same
// sweep, 16-byte vector loads, FP64 accumulation; block partials are summed
// on the device so only the final coefficients cross to the host.
#pragma once
#include <cuda_runtime.h>

namespace rism {

constexpr int kVecMax = 32;

template <typename T> struct VecSet {
  const T *p[kVecMax];
};
struct Coefs {
  double c[kVecMax];
};

template <typename T> struct Wide;
template <> struct Wide<float> { using type = float4; static constexpr int n = 4; };
template <> struct Wide<double> { using type = double2; static constexpr int n = 2; };

// The dot sweep of thread `i0` (stride `st`) over nw wide elements:
// acc[v] += w . V_v for v < nv.  NVT (>= nv) bounds the accumulators held in
// registers; for NVT <= 4 two strided elements are loaded before either is
// used, so a thread keeps twice the bytes in flight.  The accumulation order
// is that of the plain strided loop for every NVT.
template <typename T, int NVT>
__device__ __forceinline__ void mdot_sweep(long long nw, long long i0, long long st, const T *__restrict__ w, int nv,
                                           const VecSet<T> &vs, double *acc) {
  using VT = typename Wide<T>::type;
  constexpr int WN = Wide<T>::n;
  constexpr int U = NVT <= 4 ? 2 : 1;
  for (long long i = i0; i < nw; i += U * st) {
    VT a[U], b[U][NVT];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long iu = i + u * st;
      if (iu < nw) {
        a[u] = reinterpret_cast<const VT *>(w)[iu];
#pragma unroll
        for (int v = 0; v < NVT; ++v)
          if (v < nv) b[u][v] = reinterpret_cast<const VT *>(vs.p[v])[iu];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (i + u * st < nw) {
        const T *ar = reinterpret_cast<const T *>(&a[u]);
#pragma unroll
        for (int v = 0; v < NVT; ++v) {
          if (v < nv) {
            const T *br = reinterpret_cast<const T *>(&b[u][v]);
            // products in the basis precision, one conversion per vector load
            // (float -> double conversions would otherwise bound the kernel)
            T s = T(0);
#pragma unroll
            for (int q = 0; q < WN; ++q) s += ar[q] * br[q];
            acc[v] += (double)s;
          }
        }
      }
    }
  }
}

// part[b * kVecMax + v] = sum over block b's range of w . V_v  (v < nv <= NVT)
template <typename T, int NVT = kVecMax>
__global__ void __launch_bounds__(256) k_mdotv(long long nw, const T *__restrict__ w, int nv, VecSet<T> vs,
                                              double *__restrict__ part) {
  double acc[NVT];
#pragma unroll
  for (int v = 0; v < NVT; ++v) acc[v] = 0.0;
  mdot_sweep<T, NVT>(nw, (long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x, w, nv,
                     vs, acc);
  __shared__ double sm[NVT][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NVT; ++v) {
    if (v < nv) {
      double a = acc[v];
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0) sm[v][wid] = a;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < nv) {
    double a = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a += sm[threadIdx.x][q];
    part[(long long)blockIdx.x * kVecMax + threadIdx.x] = a;
  }
}

// w = ws * w - sum_v c_v V_v; part[b] = block b's sum of w^2 (if part).
// c_v = cf.c[v], times dcoef[v] when dcoef (device-resident coefficients,
// e.g. dot products reduced on the device) is given.  NVT (>= nv) bounds the
// basis vectors held in registers; a thread loads U strided wide elements of
// every operand before it uses any, so small updates still keep enough bytes
// in flight to stream at HBM rate.  w is not read when ws == 0 and not
// written back when the call only measures it (nv == 0, ws == 1).  The
// arithmetic and the accumulation order are those of the plain strided loop.
template <typename T, int NVT = kVecMax>
__global__ void __launch_bounds__(256) k_maxpyv(long long nw, T *__restrict__ w, double ws, int nv, VecSet<T> vs,
                                               Coefs cf, const double *__restrict__ dcoef,
                                               double *__restrict__ part) {
  using VT = typename Wide<T>::type;
  constexpr int WN = Wide<T>::n;
  constexpr int U = NVT <= 2 ? 4 : (NVT <= 8 ? 2 : 1);
  // the update runs in the basis precision; coefficients converted once
  T c[NVT];
#pragma unroll
  for (int v = 0; v < NVT; ++v) c[v] = (T)(dcoef ? (v < nv ? cf.c[v] * dcoef[v] : 0.0) : cf.c[v]);
  const T wsT = (T)ws;
  const bool rd = ws != 0.0, wr = !(nv == 0 && ws == 1.0);
  const long long st = (long long)gridDim.x * blockDim.x;
  double s2 = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += U * st) {
    VT a[U], b[U][NVT];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long iu = i + u * st;
      if (iu < nw) {
        if (rd) a[u] = reinterpret_cast<const VT *>(w)[iu];
#pragma unroll
        for (int v = 0; v < NVT; ++v)
          if (v < nv) b[u][v] = reinterpret_cast<const VT *>(vs.p[v])[iu];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long iu = i + u * st;
      if (iu < nw) {
        const T *ar = reinterpret_cast<const T *>(&a[u]);
        VT o;
        T *r = reinterpret_cast<T *>(&o);
#pragma unroll
        for (int q = 0; q < WN; ++q) r[q] = rd ? wsT * ar[q] : T(0);
#pragma unroll
        for (int v = 0; v < NVT; ++v) {
          if (v < nv) {
            const T *br = reinterpret_cast<const T *>(&b[u][v]);
#pragma unroll
            for (int q = 0; q < WN; ++q) r[q] -= c[v] * br[q];
          }
        }
        T sq = T(0);
#pragma unroll
        for (int q = 0; q < WN; ++q) sq += r[q] * r[q];
        s2 += (double)sq;
        if (wr) reinterpret_cast<VT *>(w)[iu] = o;
      }
    }
  }
  if (part) {
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    __shared__ double sm[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sm[wid] = s2;
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a += sm[q];
      part[blockIdx.x] = a;
    }
  }
}

// out[v] = sum_b part[b * stride + v] for v < nv (<= kVecMax): one block of
// kColsumThreads as (v, group) lanes, lanes = the power of two >= nv; group
// q sums every groups-th partial, then a pairwise tree over the groups (a
// fixed order).  With few vectors most of the block's threads take part
// instead of eight per vector.
constexpr int kColsumThreads = 1024;
__global__ static void __launch_bounds__(kColsumThreads) k_colsum(int nblk, int stride, int nv,
                                                                 const double *__restrict__ part,
                                                                 double *__restrict__ out) {
  __shared__ double red[kColsumThreads];
  int lanes = 1;
  while (lanes < nv) lanes <<= 1;
  const int groups = kColsumThreads / lanes;
  const int t = threadIdx.x, v = t % lanes, q = t / lanes;
  double a = 0.0;
  if (v < nv)
#pragma unroll 4
    for (int b = q; b < nblk; b += groups) a += part[(long long)b * stride + v];
  red[t] = a;
  __syncthreads();
  for (int st = kColsumThreads / 2; st >= lanes; st >>= 1) {
    if (t < st) red[t] += red[t + st];
    __syncthreads();
  }
  if (t < nv) out[t] = red[t];
}

// w /= sqrt(*nrm2) (w = 0 when the norm is 0); the norm goes to *hout.
// Used by the device-driven GMRES, whose basis is normalised explicitly.
template <typename T>
__global__ void k_scale_norm(long long n, T *__restrict__ w, const double *__restrict__ nrm2,
                             double *__restrict__ hout) {
  const double s = sqrt(fmax(*nrm2, 0.0));
  if (hout && blockIdx.x == 0 && threadIdx.x == 0) *hout = s;
  const T inv = s > 0.0 ? (T)(1.0 / s) : T(0);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    w[i] *= inv;
}

// The sweeps of the device-driven GMRES with their reductions fused in: the
// last block to finish a sweep (an atomic ticket, reset for the next graph
// replay) sums the block partials in a fixed order.
//
// k_mdot_red: h[v] = w . V_v for v < nv.
template <typename T, int NVT = kVecMax>
__global__ void __launch_bounds__(256) k_mdot_red(long long nw, const T *__restrict__ w, int nv, VecSet<T> vs,
                                                 double *__restrict__ part, unsigned *__restrict__ ticket,
                                                 double *__restrict__ h) {
  double acc[NVT];
#pragma unroll
  for (int v = 0; v < NVT; ++v) acc[v] = 0.0;
  mdot_sweep<T, NVT>(nw, (long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x, w, nv,
                     vs, acc);
  __shared__ double sm[NVT][8];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NVT; ++v) {
    if (v < nv) {
      double a = acc[v];
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0) sm[v][wid] = a;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < nv) {
    double a = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a += sm[threadIdx.x][q];
    part[(long long)blockIdx.x * kVecMax + threadIdx.x] = a;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double red[8][kVecMax];
  const int v = threadIdx.x % kVecMax, j = threadIdx.x / kVecMax;  // 256 threads: 8 x 32
  double s = 0.0;
  if (v < nv)
    for (int b = j; b < (int)gridDim.x; b += 8) s += part[(long long)b * kVecMax + v];
  red[j][v] = s;
  __syncthreads();
  if (j == 0 && v < nv) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += red[q][v];
    h[v] = t;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// k_maxpy_red: w -= sum_v h_v V_v (v < nv) and *hn = |w| reduced likewise.
template <typename T>
__global__ void __launch_bounds__(256) k_maxpy_red(long long nw, T *__restrict__ w, int nv, VecSet<T> vs,
                                                  const double *__restrict__ h, double *__restrict__ part,
                                                  unsigned *__restrict__ ticket, double *__restrict__ hn) {
  using VT = typename Wide<T>::type;
  constexpr int WN = Wide<T>::n;
  T c[kVecMax];
#pragma unroll
  for (int v = 0; v < kVecMax; ++v) c[v] = (T)(v < nv ? h[v] : 0.0);
  double s2 = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += (long long)gridDim.x * blockDim.x) {
    const VT a = reinterpret_cast<const VT *>(w)[i];
    const T *ar = reinterpret_cast<const T *>(&a);
    VT o;
    T *r = reinterpret_cast<T *>(&o);
#pragma unroll
    for (int q = 0; q < WN; ++q) r[q] = ar[q];
#pragma unroll
    for (int v = 0; v < kVecMax; ++v) {
      if (v < nv) {
        const VT b = reinterpret_cast<const VT *>(vs.p[v])[i];
        const T *br = reinterpret_cast<const T *>(&b);
#pragma unroll
        for (int q = 0; q < WN; ++q) r[q] -= c[v] * br[q];
      }
    }
    T sq = T(0);
#pragma unroll
    for (int q = 0; q < WN; ++q) sq += r[q] * r[q];
    s2 += (double)sq;
    reinterpret_cast<VT *>(w)[i] = o;
  }
  __shared__ double sm[8];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if (lane == 0) sm[wid] = s2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a += sm[q];
    part[blockIdx.x] = a;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double red[256];
  double s = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += part[b];
  red[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)blockDim.x; ++q) t += red[q];
    *hn = sqrt(t);
    *ticket = 0u;
  }
}

// w /= *hn (w = 0 when it is 0).
template <typename T> __global__ void k_scale_by(long long n, T *__restrict__ w, const double *__restrict__ hn) {
  const double s = *hn;
  const T inv = s > 0.0 ? (T)(1.0 / s) : T(0);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    w[i] *= inv;
}

// Least squares of a k-step Arnoldi run, on one thread: min |beta e1 - H y|
// with H's column j at H[j * (k + 1) + i], i <= j + 1; then y[0] += beta,
// so that sum y_j V_j = x + r0 (the GMRES iterate plus its right-hand side).
__global__ static void k_arnoldi_lsq(int k, const double *__restrict__ H, const double *__restrict__ beta,
                                     double *__restrict__ y) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double R[kVecMax][kVecMax + 1];  // R[i][j], i <= j + 1
  double g[kVecMax + 1], cs[kVecMax], sn[kVecMax];
  for (int j = 0; j < k; ++j)
    for (int i = 0; i <= j + 1; ++i) R[i][j] = H[j * (k + 1) + i];
  for (int i = 0; i <= k; ++i) g[i] = 0.0;
  g[0] = *beta;
  for (int j = 0; j < k; ++j) {
    for (int i = 0; i < j; ++i) {
      const double a = R[i][j], b = R[i + 1][j];
      R[i][j] = cs[i] * a + sn[i] * b;
      R[i + 1][j] = -sn[i] * a + cs[i] * b;
    }
    const double a = R[j][j], b = R[j + 1][j];
    const double r = hypot(a, b);
    cs[j] = r == 0.0 ? 1.0 : a / r;
    sn[j] = r == 0.0 ? 0.0 : b / r;
    R[j][j] = r;
    g[j + 1] = -sn[j] * g[j];
    g[j] = cs[j] * g[j];
  }
  for (int i = k - 1; i >= 0; --i) {
    double s = g[i];
    for (int l = i + 1; l < k; ++l) s -= R[i][l] * y[l];
    y[i] = R[i][i] != 0.0 ? s / R[i][i] : 0.0;
  }
  if (k > 0) y[0] += *beta;
}

// Launch of the dot sweeps with the smallest accumulator bound NVT >= nv.
template <typename T>
void launch_mdotv(unsigned grid, cudaStream_t st, long long nw, const T *w, int nv, const VecSet<T> &vs,
                  double *part) {
  if (nv <= 1) k_mdotv<T, 1><<<grid, 256, 0, st>>>(nw, w, nv, vs, part);
  else if (nv <= 2) k_mdotv<T, 2><<<grid, 256, 0, st>>>(nw, w, nv, vs, part);
  else if (nv <= 4) k_mdotv<T, 4><<<grid, 256, 0, st>>>(nw, w, nv, vs, part);
  else if (nv <= 8) k_mdotv<T, 8><<<grid, 256, 0, st>>>(nw, w, nv, vs, part);
  else if (nv <= 16) k_mdotv<T, 16><<<grid, 256, 0, st>>>(nw, w, nv, vs, part);
  else k_mdotv<T, kVecMax><<<grid, 256, 0, st>>>(nw, w, nv, vs, part);
}
// Launch of the update with the smallest basis bound NVT >= nv.
template <typename T>
void launch_maxpyv(unsigned grid, cudaStream_t st, long long nw, T *w, double ws, int nv, const VecSet<T> &vs,
                   const Coefs &cf, const double *dcoef, double *part) {
  if (nv <= 1) k_maxpyv<T, 1><<<grid, 256, 0, st>>>(nw, w, ws, nv, vs, cf, dcoef, part);
  else if (nv <= 2) k_maxpyv<T, 2><<<grid, 256, 0, st>>>(nw, w, ws, nv, vs, cf, dcoef, part);
  else if (nv <= 4) k_maxpyv<T, 4><<<grid, 256, 0, st>>>(nw, w, ws, nv, vs, cf, dcoef, part);
  else if (nv <= 8) k_maxpyv<T, 8><<<grid, 256, 0, st>>>(nw, w, ws, nv, vs, cf, dcoef, part);
  else if (nv <= 16) k_maxpyv<T, 16><<<grid, 256, 0, st>>>(nw, w, ws, nv, vs, cf, dcoef, part);
  else k_maxpyv<T, kVecMax><<<grid, 256, 0, st>>>(nw, w, ws, nv, vs, cf, dcoef, part);
}
template <typename T>
void launch_mdot_red(unsigned grid, cudaStream_t st, long long nw, const T *w, int nv, const VecSet<T> &vs,
                     double *part, unsigned *ticket, double *h) {
  if (nv <= 1) k_mdot_red<T, 1><<<grid, 256, 0, st>>>(nw, w, nv, vs, part, ticket, h);
  else if (nv <= 2) k_mdot_red<T, 2><<<grid, 256, 0, st>>>(nw, w, nv, vs, part, ticket, h);
  else if (nv <= 4) k_mdot_red<T, 4><<<grid, 256, 0, st>>>(nw, w, nv, vs, part, ticket, h);
  else if (nv <= 8) k_mdot_red<T, 8><<<grid, 256, 0, st>>>(nw, w, nv, vs, part, ticket, h);
  else if (nv <= 16) k_mdot_red<T, 16><<<grid, 256, 0, st>>>(nw, w, nv, vs, part, ticket, h);
  else k_mdot_red<T, kVecMax><<<grid, 256, 0, st>>>(nw, w, nv, vs, part, ticket, h);
}

}  // namespace rism
