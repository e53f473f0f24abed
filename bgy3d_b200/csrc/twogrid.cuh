// Grid-transfer kernels of the two-grid preconditioner.
//
// Restriction and prolongation between the fine grid (N points per axis)
// and a coarse grid (Nc points) of the same periodic box, both with points
// i * L / n - L / 2, are band-limited (spectral) transfers.  Per axis
//
//   R[i][j] = (1/N) sum_{|k| <= Nc/2} w_k cos(2 pi k (i/Nc - j/N)),
//   P[j][i] = (N/Nc) R[i][j],
//
// with w_k = 1/2 at |k| = Nc/2 for even Nc and 1 otherwise: R keeps the
// Fourier modes both grids resolve, P interpolates them back.  Both are
// separable, so a 3D transfer is three dense matrix sweeps, one per axis;
// the x sweep (the one that touches the full fine field) is a small
// register-tiled matrix product streamed once over HBM.
#pragma once
#include <cuda_runtime.h>

namespace tg {

// Restriction along x: out[row][i] = s * sum_j R[i][j] in[row][j]
// (rows x N0 -> rows x Nc0), R given transposed: Rt[j][i] = R[i][j].
// CTA tile 128 rows x 48 coarse columns, 128 threads, 8 x 6 outputs per
// thread, K staged through shared memory in chunks of 32; rows are padded to
// a multiple of 4 floats so a thread's 8 rows load as two float4 and its 6
// columns as three float2 (48 FMA per 5 shared loads).
constexpr int kRxRows = 128, kRxCols = 48, kRxK = 32, kRxThreads = 128, kRxPad = kRxRows + 4;

template <typename TI>
__global__ void __launch_bounds__(kRxThreads) k_restrict_x(long long rows, int N, int Nc, const TI *__restrict__ in,
                                                          float s, const float *__restrict__ Rt,
                                                          float *__restrict__ out) {
  __shared__ __align__(16) float Xs[kRxK][kRxPad];
  __shared__ __align__(16) float Rs[kRxK][kRxCols];
  const int t = threadIdx.x;
  const int tr = t >> 3, tc = t & 7;  // rows tr*8.., cols tc*6..
  const long long row0 = (long long)blockIdx.x * kRxRows;
  const int col0 = blockIdx.y * kRxCols;
  float acc[8][6];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 6; ++b) acc[a][b] = 0.f;
  for (int k0 = 0; k0 < N; k0 += kRxK) {
    // X chunk: 128 rows x 32 k; a warp reads 32 consecutive k of one row
    for (int q = 0; q < kRxRows / 4; ++q) {
      const int r = q * 4 + (t >> 5), kk = t & 31;
      const long long row = row0 + r;
      float v = 0.f;
      if (row < rows && k0 + kk < N) v = (float)in[row * N + k0 + kk];
      Xs[kk][r] = v;
    }
    for (int e = t; e < kRxK * kRxCols; e += kRxThreads) {
      const int kk = e / kRxCols, cc = e % kRxCols;
      Rs[kk][cc] = (col0 + cc < Nc && k0 + kk < N) ? Rt[(long long)(k0 + kk) * Nc + col0 + cc] : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kRxK; ++kk) {
      const float4 x0 = *reinterpret_cast<const float4 *>(&Xs[kk][tr * 8]);
      const float4 x1 = *reinterpret_cast<const float4 *>(&Xs[kk][tr * 8 + 4]);
      const float2 r0 = *reinterpret_cast<const float2 *>(&Rs[kk][tc * 6]);
      const float2 r1 = *reinterpret_cast<const float2 *>(&Rs[kk][tc * 6 + 2]);
      const float2 r2 = *reinterpret_cast<const float2 *>(&Rs[kk][tc * 6 + 4]);
      const float x[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
      const float r[6] = {r0.x, r0.y, r1.x, r1.y, r2.x, r2.y};
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 6; ++b) acc[a][b] = fmaf(x[a], r[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const long long row = row0 + tr * 8 + a;
    if (row >= rows) continue;
#pragma unroll
    for (int b = 0; b < 6; ++b) {
      const int col = col0 + tc * 6 + b;
      if (col < Nc) out[row * Nc + col] = s * acc[a][b];
    }
  }
}

// Prolongation along x with the residual term of the preconditioner:
// out[row][j] = sum_i P[j][i] y[row][i] - s * r[row][j]
// (rows x Nc0 -> rows x N0), P given transposed: Pt[i][j] = P[j][i].
// CTA tile 64 rows x 128 fine columns, 128 threads, 8 x 8 outputs per
// thread (64 FMA per four float4 shared loads); each thread reads r and
// writes out as 8 consecutive elements of a row, a warp 16 x 8 of them.
constexpr int kPxRows = 64, kPxCols = 128, kPxK = 16, kPxThreads = 128, kPxPad = kPxRows + 4;

template <typename T> struct Vec8;
template <> struct Vec8<float> {
  __device__ __forceinline__ static void load(const float *p, float v[8]) {
    const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  }
  __device__ __forceinline__ static void store(float *p, const float v[8]) {
    reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4 *>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
  }
};
template <> struct Vec8<double> {
  __device__ __forceinline__ static void load(const double *p, double v[8]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 a = reinterpret_cast<const double2 *>(p)[q];
      v[2 * q] = a.x; v[2 * q + 1] = a.y;
    }
  }
  __device__ __forceinline__ static void store(double *p, const double v[8]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) reinterpret_cast<double2 *>(p)[q] = make_double2(v[2 * q], v[2 * q + 1]);
  }
};

template <typename TO, typename TR>
__global__ void __launch_bounds__(kPxThreads) k_prolong_x(long long rows, int N, int Nc, const float *__restrict__ y,
                                                         const float *__restrict__ Pt, const TR *__restrict__ r,
                                                         double s, TO *__restrict__ out) {
  __shared__ __align__(16) float Ys[kPxK][kPxPad];
  __shared__ __align__(16) float Ps[kPxK][kPxCols];
  const int t = threadIdx.x;
  const int tr = t >> 4, tc = t & 15;  // rows tr*8.., cols tc*8..
  const long long row0 = (long long)blockIdx.x * kPxRows;
  const int col0 = blockIdx.y * kPxCols;
  float acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;
  for (int k0 = 0; k0 < Nc; k0 += kPxK) {
    for (int e = t; e < kPxK * kPxRows; e += kPxThreads) {
      const int rr = e / kPxK, kk = e % kPxK;
      const long long row = row0 + rr;
      Ys[kk][rr] = (row < rows && k0 + kk < Nc) ? y[row * Nc + k0 + kk] : 0.f;
    }
    for (int e = t; e < kPxK * kPxCols; e += kPxThreads) {
      const int kk = e / kPxCols, cc = e % kPxCols;
      Ps[kk][cc] = (col0 + cc < N && k0 + kk < Nc) ? Pt[(long long)(k0 + kk) * N + col0 + cc] : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kPxK; ++kk) {
      const float4 y0 = *reinterpret_cast<const float4 *>(&Ys[kk][tr * 8]);
      const float4 y1 = *reinterpret_cast<const float4 *>(&Ys[kk][tr * 8 + 4]);
      const float4 p0 = *reinterpret_cast<const float4 *>(&Ps[kk][tc * 8]);
      const float4 p1 = *reinterpret_cast<const float4 *>(&Ps[kk][tc * 8 + 4]);
      const float yv[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
      const float pv[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(yv[a], pv[b], acc[a][b]);
    }
    __syncthreads();
  }
  const int c0 = col0 + tc * 8;
  const bool full = c0 + 8 <= N && (N % 8) == 0;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const long long row = row0 + tr * 8 + a;
    if (row >= rows) continue;
    const long long p = row * N + c0;
    if (full) {
      TR rv[8];
      TO ov[8];
      Vec8<TR>::load(r + p, rv);
#pragma unroll
      for (int b = 0; b < 8; ++b) ov[b] = (TO)((double)acc[a][b] - s * (double)rv[b]);
      Vec8<TO>::store(out + p, ov);
    } else {
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (c0 + b < N) out[p + b] = (TO)((double)acc[a][b] - s * (double)r[p + b]);
    }
  }
}

// Transfer along a strided axis: out[o][j][i] = sum_k A[j][k] in[o][k][i]
// for o < outer, j < n_out, k < n_in <= 512, i < inner (i contiguous).
// Each thread owns one (o, i) and 8 consecutive j (blockIdx.y selects the
// 8-row slab of A, staged transposed in shared memory).
constexpr int kAxJ = 8, kAxThreads = 256, kAxMaxIn = 512;

__global__ void __launch_bounds__(kAxThreads) k_transfer_axis(int outer, int n_in, int n_out, int inner,
                                                             const float *__restrict__ in,
                                                             const float *__restrict__ A,
                                                             float *__restrict__ out) {
  __shared__ __align__(16) float At[kAxMaxIn][kAxJ];
  const int j0 = blockIdx.y * kAxJ;
  for (int e = threadIdx.x; e < n_in * kAxJ; e += kAxThreads) {
    const int k = e / kAxJ, jj = e % kAxJ;
    At[k][jj] = (j0 + jj < n_out) ? A[(long long)(j0 + jj) * n_in + k] : 0.f;
  }
  __syncthreads();
  const long long p = (long long)blockIdx.x * kAxThreads + threadIdx.x;
  if (p >= (long long)outer * inner) return;
  const int o = (int)(p / inner), i = (int)(p % inner);
  const float *src = in + (long long)o * n_in * inner + i;
  float acc[kAxJ];
#pragma unroll
  for (int jj = 0; jj < kAxJ; ++jj) acc[jj] = 0.f;
#pragma unroll 4
  for (int k = 0; k < n_in; ++k) {
    const float v = src[(long long)k * inner];
    const float4 a0 = *reinterpret_cast<const float4 *>(&At[k][0]);
    const float4 a1 = *reinterpret_cast<const float4 *>(&At[k][4]);
    acc[0] = fmaf(a0.x, v, acc[0]); acc[1] = fmaf(a0.y, v, acc[1]);
    acc[2] = fmaf(a0.z, v, acc[2]); acc[3] = fmaf(a0.w, v, acc[3]);
    acc[4] = fmaf(a1.x, v, acc[4]); acc[5] = fmaf(a1.y, v, acc[5]);
    acc[6] = fmaf(a1.z, v, acc[6]); acc[7] = fmaf(a1.w, v, acc[7]);
  }
  float *dst = out + (long long)o * n_out * inner + i;
#pragma unroll
  for (int jj = 0; jj < kAxJ; ++jj)
    if (j0 + jj < n_out) dst[(long long)(j0 + jj) * inner] = acc[jj];
}

// The same product with J outputs per thread, A's J-row slab staged
// transposed in dynamic shared memory ([n_in][J] floats): wider slabs read
// the input fewer times (n_out / J instead of n_out / 8).
template <int J>
__global__ void __launch_bounds__(kAxThreads) k_transfer_axis_j(int outer, int n_in, int n_out, int inner,
                                                              const float *__restrict__ in,
                                                              const float *__restrict__ A,
                                                              float *__restrict__ out) {
  extern __shared__ __align__(16) float AtJ[];
  const int j0 = blockIdx.y * J;
  for (int e = threadIdx.x; e < n_in * J; e += kAxThreads) {
    const int k = e / J, jj = e % J;
    AtJ[e] = (j0 + jj < n_out) ? A[(long long)(j0 + jj) * n_in + k] : 0.f;
  }
  __syncthreads();
  const long long p = (long long)blockIdx.x * kAxThreads + threadIdx.x;
  if (p >= (long long)outer * inner) return;
  const int o = (int)(p / inner), i = (int)(p % inner);
  const float *src = in + (long long)o * n_in * inner + i;
  float acc[J];
#pragma unroll
  for (int jj = 0; jj < J; ++jj) acc[jj] = 0.f;
  // 8 strided input loads in flight per thread (the sweep is bound by their
  // latency, not by the FMAs)
#pragma unroll 8
  for (int k = 0; k < n_in; ++k) {
    const float v = src[(long long)k * inner];
    const float4 *a = reinterpret_cast<const float4 *>(&AtJ[k * J]);
#pragma unroll
    for (int q = 0; q < J / 4; ++q) {
      const float4 w = a[q];
      acc[4 * q] = fmaf(w.x, v, acc[4 * q]);
      acc[4 * q + 1] = fmaf(w.y, v, acc[4 * q + 1]);
      acc[4 * q + 2] = fmaf(w.z, v, acc[4 * q + 2]);
      acc[4 * q + 3] = fmaf(w.w, v, acc[4 * q + 3]);
    }
  }
  float *dst = out + (long long)o * n_out * inner + i;
#pragma unroll
  for (int jj = 0; jj < J; ++jj)
    if (j0 + jj < n_out) dst[(long long)(j0 + jj) * inner] = acc[jj];
}

}  // namespace tg
