// fft_static.cuh -- compile-time-length FFT building blocks and TMA helpers
// for the shape-specialised passes (sm_100a).
//
// A length-N transform of a shared-memory tile is done as N = R1 * R2 in two
// register steps (four-step / Cooley-Tukey): step 1 runs R2 * ncol DFTs of
// length R1 (stride R2) in registers and writes them back in place with the
// W_N^(n2 k1) twiddles applied; step 2 runs R1 * ncol DFTs of length R2 on
// contiguous runs and writes the outputs to their natural positions.  The
// register DFTs are composed at compile time from radix 4, 2 and 3, so every
// index is a constant.  256 = 16 x 16 costs two shared-memory round trips
// instead of four radix-4 Stockham stages.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_core.cuh"

namespace rism {

// a * W_R^q with compile-time-foldable q (after unrolling): the quarter
// turns are exact, the rest come from the table tw[j] = W_NT^j, stride = NT/R.
template <int R, bool INV, typename V>
__device__ __forceinline__ V tmul(V a, int q, const V *tw, int stride) {
  q %= R;
  if (q == 0) return a;
  if (4 * q == R) return cmuli<INV>(a);
  if (2 * q == R) { a.x = -a.x; a.y = -a.y; return a; }
  if (4 * q == 3 * R) return cmuli<!INV>(a);
  V t = tw[q * stride];
  if (INV) t.y = -t.y;
  return cmul(a, t);
}

// In-register DFT of compile-time length R (forward exp(-2 pi i n k / R)).
template <int R, bool INV, typename V> struct RDft {
  static constexpr int P = (R % 4 == 0) ? 4 : ((R % 2 == 0) ? 2 : 3);
  static constexpr int Q = R / P;
  __device__ __forceinline__ static void run(V *a, const V *tw, int stride) {
    V t[R];
#pragma unroll
    for (int n2 = 0; n2 < Q; ++n2) {
      V u[P];
#pragma unroll
      for (int n1 = 0; n1 < P; ++n1) u[n1] = a[Q * n1 + n2];
      RDft<P, INV, V>::run(u, tw, stride * Q);
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) t[k1 * Q + n2] = tmul<R, INV>(u[k1], n2 * k1, tw, stride);
    }
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      V u[Q];
#pragma unroll
      for (int n2 = 0; n2 < Q; ++n2) u[n2] = t[k1 * Q + n2];
      RDft<Q, INV, V>::run(u, tw, stride * P);
#pragma unroll
      for (int k2 = 0; k2 < Q; ++k2) a[k1 + P * k2] = u[k2];
    }
  }
};
template <bool INV, typename V> struct RDft<1, INV, V> {
  __device__ __forceinline__ static void run(V *, const V *, int) {}
};
template <bool INV, typename V> struct RDft<2, INV, V> {
  __device__ __forceinline__ static void run(V *a, const V *, int) { Butterfly<2, INV, V>::run(a); }
};
template <bool INV, typename V> struct RDft<3, INV, V> {
  __device__ __forceinline__ static void run(V *a, const V *, int) { Butterfly<3, INV, V>::run(a); }
};
template <bool INV, typename V> struct RDft<4, INV, V> {
  __device__ __forceinline__ static void run(V *a, const V *, int) { Butterfly<4, INV, V>::run(a); }
};

// First-step radix of a compile-time length: the largest of 16, 8, 12, 6, 4
// dividing N with a cofactor no larger than it (16 for 512).
template <int N> struct Split {
  static constexpr int R1 = N == 512 ? 16  // 16 x 32: the second step holds 32 points per thread
                          : (N % 16 == 0 && N / 16 <= 16) ? 16
                          : (N % 8 == 0 && N / 8 <= 8) ? 8
                          : (N % 12 == 0 && N / 12 <= 12) ? 12
                          : (N % 6 == 0 && N / 6 <= 8) ? 6 : 4;
  static constexpr int R2 = N / R1;
};

// A split with R1 near sqrt(N) (64 = 8 x 8, 96 = 12 x 8): where a tile has
// few columns, Split's larger first radix leaves most threads of a step idle
// (16 x 4 over 16 columns: 64 DFTs for 256 threads) and holds twice the
// values per thread.
template <int N> struct SplitSq {
  static constexpr int R1 = N == 48 ? 8 : N == 64 ? 8 : N == 72 ? 8 : N == 96 ? 12 : N == 128 ? 16 : Split<N>::R1;
  static constexpr int R2 = N / R1;
};

// The split of the row-batched transforms (x passes and x transfers: one
// work item per row and index, COLFAST false), where Split's larger first
// radix would leave most of the CTA idle in one step (32 = 16 x 2 gives R2 x
// rows items of 16-point DFTs); here both steps keep the CTA busy.
template <int N> struct SplitRow {
  static constexpr int R1 = N == 24 ? 6 : N == 32 ? 8 : N == 36 ? 6 : N == 48 ? 8 : N == 96 ? 12 : Split<N>::R1;
  static constexpr int R2 = N / R1;
};

// Tile layouts: element (i, col) of the transform index i and column col.
// Columns fastest, [n][B] tiles of NB per sub-tile stacked SB times
// ([s][n][b], the TMA boxes of the y and z passes):
template <int N, int B> struct LayCol {
  __device__ __forceinline__ static int at(int i, int col) { return (col / B) * (N * B) + i * B + (col % B); }
};
// Rows of N with one pad element every R2 (the x pass), keeping the strided
// accesses of both steps off a single bank, and the row stride RS = R2 mod
// 16 complex values: in step 1 a warp spans 32 / R2 rows of R2 consecutive
// work items each, which then fall on disjoint banks instead of piling onto
// the same ones (a stride that is a multiple of 32 banks made 128-point rows
// 4-way conflicted).
template <int N, int R2> struct LayRow {
  static constexpr int RS0 = N + N / R2;
  static constexpr int RS = RS0 + ((R2 % 16) - RS0 % 16 + 16) % 16;
  __device__ __forceinline__ static int at(int i, int row) { return row * RS + i + i / R2; }
};

// Two-step transform of NCOL columns of length N by NTHR threads (tid <
// NTHR; threads with act false only take part in the barriers, so several
// groups of one CTA can transform their own tiles together).  COLFAST maps
// consecutive threads to consecutive columns (column-contiguous tiles),
// otherwise to consecutive transform indices (row-contiguous tiles).  Ends
// synchronised.
template <int N, int NCOL, int NTHR, bool INV, bool COLFAST, class Lay, class S = Split<N>, typename V>
__device__ __forceinline__ void fft2g(V *buf, const V *tw, int tid, bool act) {
  constexpr int R1 = S::R1, R2 = S::R2;
  static_assert(R1 * R2 == N, "split must factor N");
  constexpr int I1 = R2 * NCOL;
#pragma unroll
  for (int it = 0; it < (I1 + NTHR - 1) / NTHR; ++it) {
    const int w = tid + it * NTHR;
    if (act && (I1 % NTHR == 0 || w < I1)) {
      const int col = COLFAST ? w % NCOL : w / R2;
      const int n2 = COLFAST ? w / NCOL : w % R2;
      V u[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) u[n1] = buf[Lay::at(R2 * n1 + n2, col)];
      RDft<R1, INV, V>::run(u, tw, N / R1);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        V x = u[k1];
        if (k1 != 0 && n2 != 0) {
          V t = tw[n2 * k1];
          if (INV) t.y = -t.y;
          x = cmul(x, t);
        }
        buf[Lay::at(R2 * k1 + n2, col)] = x;
      }
    }
  }
  __syncthreads();
  constexpr int I2 = R1 * NCOL;
  constexpr int C2 = (I2 + NTHR - 1) / NTHR;
  V u[C2][R2];
#pragma unroll
  for (int it = 0; it < C2; ++it) {
    const int w = tid + it * NTHR;
    if (act && (I2 % NTHR == 0 || w < I2)) {
      const int col = COLFAST ? w % NCOL : w / R1;
      const int k1 = COLFAST ? w / NCOL : w % R1;
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) u[it][n2] = buf[Lay::at(R2 * k1 + n2, col)];
      RDft<R2, INV, V>::run(u[it], tw, N / R2);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < C2; ++it) {
    const int w = tid + it * NTHR;
    if (act && (I2 % NTHR == 0 || w < I2)) {
      const int col = COLFAST ? w % NCOL : w / R1;
      const int k1 = COLFAST ? w / NCOL : w % R1;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) buf[Lay::at(k1 + R1 * k2, col)] = u[it][k2];
    }
  }
  __syncthreads();
}
// The whole CTA as one group of NTHR threads.
template <int N, int NCOL, int NTHR, bool INV, bool COLFAST, class Lay, class S = Split<N>, typename V>
__device__ __forceinline__ void fft2(V *buf, const V *tw) {
  fft2g<N, NCOL, NTHR, INV, COLFAST, Lay, S>(buf, tw, (int)threadIdx.x, true);
}

// ------------------------------------------------------------- TMA + mbarrier
// d_err code of a timed-out wait in the tensor-core grid transfers
// (the passes record their pass number, the coarse solve kPkErr).
constexpr int kTcErr = 6;
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Bounded wait on the mbarrier phase: false after max_polls unsuccessful polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t max_polls) {
  for (uint32_t i = 0; i < max_polls; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// Every thread of the CTA waits for phase `parity` of `bar`; the result is
// CTA-uniform (one barrier with a vote replaces the barrier that follows the
// wait anyway).  On a timeout thread 0 records `code` in *err and waits once
// more, bounded, so that a transaction still in flight lands while the CTA
// is resident; the whole CTA then leaves together.
__device__ __forceinline__ bool cta_wait_tile(uint64_t *bar, uint32_t parity, uint32_t max_polls, int *err,
                                              int code) {
  const bool ok = mbar_wait(bar, parity, max_polls);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicExch(err, code);
      mbar_wait(bar, parity, max_polls);
    }
    __syncthreads();
    return false;
  }
  return true;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void tma_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void tma_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void tma_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace rism
