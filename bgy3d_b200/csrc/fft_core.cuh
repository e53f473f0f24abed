// fft_core.cuh -- shared-memory mixed-radix FFT building blocks for sm_100a.
//
// The 3D transforms of the 3D-RISM residual are done as batched 1D
// transforms along x, y and z.  Each CTA stages a tile of the grid in
// shared memory and runs an in-place Stockham autosort FFT on it: every
// stage reads all its butterfly inputs into registers, synchronises,
// then writes the outputs to their sorted positions, so one shared
// buffer suffices and no bit reversal is needed.  Radices 4, 2 and 3
// cover every grid size 2^a 3^b of the workloads (64..512).
//
// Element (idx, b) of a tile (idx along the transform, b the batch) is
// buf[idx * sn + b * sb].  BFAST selects how threads map to work: batch
// index fastest (tiles stored [n][batch], the y/z passes) or transform
// index fastest (tiles stored [batch][n], the x pass); either keeps the
// shared-memory accesses of a warp contiguous.
#pragma once
#include <cuda_runtime.h>

namespace rism {

template <typename T> struct Cx;
template <> struct Cx<double> { using type = double2; };
template <> struct Cx<float> { using type = float2; };

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
  V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename V> __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename V> __device__ __forceinline__ V cmuli(V a) {
  V r;
  if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}
template <typename V, typename S> __device__ __forceinline__ V cscale(V a, S s) { a.x *= s; a.y *= s; return a; }

// Longest 1D transform and stage count supported.
constexpr int kMaxN = 512;
constexpr int kMaxStages = 10;
// Registers per thread per stage: at most this many complex values (8
// doubles2 or 16 float2, i.e. 32 registers of data), so a launch must
// satisfy n * batch <= reg_complex<V>() * threads.
template <typename V> __host__ __device__ constexpr int reg_complex() { return sizeof(V) == 16 ? 8 : 16; }

// A 1D transform plan: length, radix sequence, twiddle table
// tw[q] = exp(-2 pi i q / n), q in [0, n), in the precision of the pass.
struct AxisPlan {
  int n;
  int nst;
  int rad[kMaxStages];
  const void *tw;
};

// R-point DFT in registers (forward: exp(-2 pi i r s / R)).
template <int R, bool INV, typename V> struct Butterfly;

template <bool INV, typename V> struct Butterfly<2, INV, V> {
  __device__ __forceinline__ static void run(V *a) {
    V t = a[1];
    a[1] = csub(a[0], t);
    a[0] = cadd(a[0], t);
  }
};

template <bool INV, typename V> struct Butterfly<4, INV, V> {
  __device__ __forceinline__ static void run(V *a) {
    V t0 = cadd(a[0], a[2]);
    V t1 = csub(a[0], a[2]);
    V t2 = cadd(a[1], a[3]);
    V t3 = cmuli<INV>(csub(a[1], a[3]));
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, t3);
    a[3] = csub(t1, t3);
  }
};

template <bool INV, typename V> struct Butterfly<3, INV, V> {
  __device__ __forceinline__ static void run(V *a) {
    using S = decltype(a[0].x);
    const S half = S(0.5);
    const S s3 = S(0.86602540378443864676372317075294);  // sqrt(3)/2
    V sum = cadd(a[1], a[2]);
    V dif = csub(a[1], a[2]);
    V t;
    t.x = a[0].x - half * sum.x;
    t.y = a[0].y - half * sum.y;
    V u = cscale(cmuli<INV>(dif), s3);
    a[0] = cadd(a[0], sum);
    a[1] = cadd(t, u);
    a[2] = csub(t, u);
  }
};

// One Stockham stage of radix R over the tile.  Ns = product of the radices
// of the previous stages.  Called by all threads of the CTA.
template <int R, bool INV, bool BFAST, typename V>
__device__ __forceinline__ void fft_stage(V *buf, int n, int batch, int sn, int sb, int Ns,
                                          const V *tw, int tid, int nthr) {
  constexpr int MAXIT = (reg_complex<V>() + R - 1) / R;
  const int nR = n / R;
  const int total = nR * batch;
  const int tws = n / (Ns * R);
  V a[MAXIT][R];
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int w = tid + it * nthr;
    if (w < total) {
      int j, b;
      if (BFAST) { b = w % batch; j = w / batch; } else { j = w % nR; b = w / nR; }
      const int k = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        V x = buf[(j + r * nR) * sn + b * sb];
        if (r > 0 && k > 0) {
          V t = tw[r * k * tws];
          if (INV) t.y = -t.y;
          x = cmul(x, t);
        }
        a[it][r] = x;
      }
      Butterfly<R, INV, V>::run(a[it]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int w = tid + it * nthr;
    if (w < total) {
      int j, b;
      if (BFAST) { b = w % batch; j = w / batch; } else { j = w % nR; b = w / nR; }
      const int k = j % Ns;
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[(base + r * Ns) * sn + b * sb] = a[it][r];
    }
  }
  __syncthreads();
}

// Full transform along idx for every batch column of the tile.
// Requires n * batch <= reg_complex<V>() * nthr (checked on the host).
template <bool INV, bool BFAST, typename V>
__device__ void fft_tile(V *buf, const AxisPlan &p, int batch, int sn, int sb, const V *tw) {
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  int Ns = 1;
  for (int s = 0; s < p.nst; ++s) {
    const int R = p.rad[s];
    if (R == 4)
      fft_stage<4, INV, BFAST>(buf, p.n, batch, sn, sb, Ns, tw, tid, nthr);
    else if (R == 2)
      fft_stage<2, INV, BFAST>(buf, p.n, batch, sn, sb, Ns, tw, tid, nthr);
    else
      fft_stage<3, INV, BFAST>(buf, p.n, batch, sn, sb, Ns, tw, tid, nthr);
    Ns *= R;
  }
}

}  // namespace rism
