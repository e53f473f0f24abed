// twogrid_tc.cu -- the x-axis grid transfers of the two-grid preconditioner
// on the tensor cores (sm_100a: tcgen05 MMA, accumulators in tensor memory,
// operands staged by TMA).
//
// Along x the band-limited restriction and prolongation are dense products
// of every grid row with a small table:
//
//   restriction   out[row][i] = s * sum_j R[i][j] in[row][j]    (R [Nc][N0])
//   prolongation  out[row][j] = sum_i P[j][i] y[row][i] - s r[row][j]
//                                                              (P [N0][Nc])
//
// i.e. a [rows x K] x [K x N] product (K = N0, N = Nc for R; K = Nc, N = N0
// for P) with the table as the B operand, K-major on both sides, on 128-row
// tiles (the MMA's M).  The restriction's CTA (one per SM) holds the whole
// table:
//
//   warp 0      TMA: the table once, then one 32-float K slice of the row
//               tile per pipeline stage (128-byte swizzle)
//   warps 2-5   split every stage into hi = tf32(x) (low 13 mantissa bits
//               cleared, in place) and lo = x - hi (exact in FP32)
//   warp 1      one thread issues tcgen05.mma kind::tf32: per K step
//               hi.Bhi + hi.Blo + lo.Bhi into a 128 x N FP32 accumulator
//               in tensor memory (two accumulators, alternating tiles)
//   warps 6-13  tcgen05.ld the accumulator (warp w reads lanes 32 (w % 4)
//               ..; two warps per lane quarter split the columns), scale,
//               store the rows
//
// The prolongation (k_prolong_x_tc2) gives each CTA half of every row, and
// the residual and the result move through a TMA ring (see there).
//
// The three-term split keeps the product at FP32 accuracy (the dropped
// lo.lo term is 2^-22 of the product), so the transfers agree with the FFT
// and dense forms to a few ulp.  Every mbarrier wait is bounded: a timeout
// records kTcErr in *err, raises a CTA-wide abort flag that ends every
// role's loop, and the CTA still waits (bounded) for its own copies and
// MMAs in flight before it frees the tensor memory and leaves.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "fft_static.cuh"

namespace rism {

namespace {

constexpr int kTcBM = 128;                // rows per tile: the MMA's M
constexpr int kTcKA = 32;                 // floats per K slice: one 128-byte swizzle row
constexpr int kTcWarps = 14;              // TMA, MMA, 4 split, 8 epilogue
constexpr int kTcThreads = kTcWarps * 32;
constexpr int kTcSplit0 = 2, kTcEpi0 = 6;  // first split / epilogue warp
constexpr uint32_t kTcPolls = 1u << 26;   // bounded mbarrier waits (seconds)

// The restriction's row kernel: three K slices in flight.
template <int K, int N> struct TcShape {
  static_assert(K % kTcKA == 0 && N % 32 == 0 && N <= 256, "K slices of 32 floats, N a multiple of 32 up to 256");
  static constexpr int NKA = K / kTcKA;
  static constexpr int NST = 3;
  static constexpr uint32_t A_BYTES = kTcBM * 128;  // one stage of hi (or lo)
  static constexpr uint32_t B_SLICE = N * 128;      // one K slice of the table
  static constexpr uint32_t B_BYTES = NKA * B_SLICE;
  static constexpr uint32_t OFF_BLO = B_BYTES;
  static constexpr uint32_t OFF_AHI = 2 * B_BYTES;
  static constexpr uint32_t OFF_ALO = OFF_AHI + NST * A_BYTES;
  static constexpr uint32_t OFF_BAR = OFF_ALO + NST * A_BYTES;
  // barriers: full, split, empty per stage; tmem_full[2], tmem_empty[2];
  // bfull; drain; then the tensor-memory address and the abort flag
  static constexpr int NBAR = 3 * NST + 6;
  static constexpr uint32_t OFF_MISC = OFF_BAR + NBAR * 8;
  static constexpr uint32_t SMEM = OFF_MISC + 16 + 1024;  // + alignment slack
  static constexpr uint32_t TCOLS = 2 * N <= 128 ? 128 : (2 * N <= 256 ? 256 : 512);
  // instruction descriptor: D FP32, A and B TF32, both K-major, N >> 3, M >> 4
  static constexpr uint32_t IDESC =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
};

// Shared-memory matrix descriptor of a K-major operand in the 128-byte
// swizzle layout that TMA writes: 8-row groups of 128-byte rows, 1024 bytes
// apart (SBO), layout type 2, descriptor version 1.  A K step of 8 TF32
// values inside the swizzle row adds 32 bytes (2 in the address field).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
// Arrives on `bar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
// 32 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// hi = x with the low 13 mantissa bits cleared (exactly a TF32 value), lo =
// x - hi (exact in FP32; the tensor core keeps its leading 11 bits).
__device__ __forceinline__ void tc_split4(float4 &x, float4 &lo) {
  float4 h;
  h.x = __uint_as_float(__float_as_uint(x.x) & 0xFFFFE000u);
  h.y = __uint_as_float(__float_as_uint(x.y) & 0xFFFFE000u);
  h.z = __uint_as_float(__float_as_uint(x.z) & 0xFFFFE000u);
  h.w = __uint_as_float(__float_as_uint(x.w) & 0xFFFFE000u);
  lo = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
  x = h;
}

// Bounded wait that also gives up once another role has raised the abort
// flag: 1 done, 0 timed out, -1 aborted.
__device__ __forceinline__ int tc_wait(uint64_t *bar, uint32_t parity, const volatile int *abort_flag) {
  for (uint32_t i = 0; i < kTcPolls; i += 1024) {
    if (mbar_wait(bar, parity, 1024)) return 1;
    if (*abort_flag) return -1;
  }
  return 0;
}
// The same for a whole warp (lane 0 polls); warp-uniform result.
__device__ __forceinline__ int tc_warp_wait(uint64_t *bar, uint32_t parity, const volatile int *abort_flag) {
  int r = 0;
  if ((threadIdx.x & 31) == 0) r = tc_wait(bar, parity, abort_flag);
  return __shfl_sync(0xffffffffu, r, 0);
}
__device__ __forceinline__ void tc_fail(int *err, volatile int *abort_flag) {
  atomicExch(err, kTcErr);
  *abort_flag = 1;
}

// out [rows][N] = s * in [rows][K] B^T (the restriction); tma maps the row
// data ([rows][K] FP32, box 32 x 128), tmb the table B ([N][K], box 32 x N),
// both with the 128-byte swizzle.
template <int K, int N>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_transfer_x_tc(long long rows, const __grid_constant__ CUtensorMap tma, const __grid_constant__ CUtensorMap tmb,
                    float s, float *__restrict__ out, int *__restrict__ err) {
  using S = TcShape<K, N>;
  constexpr int NST = S::NST;
  extern __shared__ unsigned char tc_raw[];
  // the swizzled tiles start on a 1024-byte boundary
  unsigned char *base = tc_raw + ((1024u - (smem_u32(tc_raw) & 1023u)) & 1023u);
  const uint32_t sb = smem_u32(base);
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + S::OFF_BAR);
  uint64_t *full = bars, *split = bars + NST, *empty = bars + 2 * NST;
  uint64_t *tfull = bars + 3 * NST, *tempty = tfull + 2, *bfull = tempty + 2, *drain = bfull + 1;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(base + S::OFF_MISC);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(base + S::OFF_MISC + 4);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ntiles = (rows + kTcBM - 1) / kTcBM;

  if (threadIdx.x == 0) {
    for (int q = 0; q < NST; ++q) {
      mbar_init(full + q, 1);
      mbar_init(split + q, kTcEpi0 - kTcSplit0);
      mbar_init(empty + q, 1);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(tfull + q, 1);
      mbar_init(tempty + q, kTcWarps - kTcEpi0);
    }
    mbar_init(bfull, 1);
    mbar_init(drain, 1);
    *abort_flag = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(S::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  // the table, once per CTA, split into hi / lo in place
  if (threadIdx.x == 0) {
    mbar_expect_tx(bfull, S::B_BYTES);
#pragma unroll 1
    for (int a = 0; a < S::NKA; ++a) tma_load_2d(base + a * S::B_SLICE, &tmb, bfull, a * kTcKA, 0);
  }
  const bool bok = mbar_wait(bfull, 0, kTcPolls);
  if (__syncthreads_or(!bok)) {
    if (threadIdx.x == 0) {
      tc_fail(err, abort_flag);
      mbar_wait(bfull, 0, kTcPolls);  // the table copies land while the CTA is resident
    }
  } else {
    float4 *bh = reinterpret_cast<float4 *>(base), *bl = reinterpret_cast<float4 *>(base + S::OFF_BLO);
    for (int i = threadIdx.x; i < (int)(S::B_BYTES / 16); i += kTcThreads) {
      float4 x = bh[i], lo;
      tc_split4(x, lo);
      bh[i] = x;
      bl[i] = lo;
    }
    fence_proxy_async();  // the generic-proxy writes, seen by the tensor core
  }
  __syncthreads();
  const bool run = *abort_flag == 0;

  if (warp == 0) {
    // ---- TMA producer: one K slice of a row tile per stage
    if (lane == 0 && run) {
      uint32_t L = 0;
      bool go = true;
      for (long long t = blockIdx.x; t < ntiles && go; t += gridDim.x) {
        for (int a = 0; a < S::NKA; ++a) {
          const uint32_t st = L % NST, n = L / NST;
          const int w = tc_wait(empty + st, (n & 1) ^ 1, abort_flag);
          if (w != 1) {
            if (w == 0) tc_fail(err, abort_flag);
            go = false;
            break;
          }
          mbar_expect_tx(full + st, S::A_BYTES);
          tma_load_2d(base + S::OFF_AHI + st * S::A_BYTES, &tma, full + st, a * kTcKA, (int)(t * kTcBM));
          ++L;
        }
      }
      // every copy issued lands before the CTA leaves (phase n of stage st
      // is the last one issued there)
      for (uint32_t st = 0; st < (uint32_t)NST; ++st)
        if (L > st) mbar_wait(full + st, ((L - 1 - st) / NST) & 1, kTcPolls);
    }
  } else if (warp == 1) {
    // ---- MMA issuer: hi.Bhi + hi.Blo + lo.Bhi per K step of 8
    if (lane == 0 && run) {
      uint32_t L = 0;
      bool go = true;
      int it = 0;
      for (long long t = blockIdx.x; t < ntiles && go; t += gridDim.x, ++it) {
        const int b = it & 1;
        const uint32_t u = (uint32_t)it >> 1;
        int w = tc_wait(tempty + b, (u & 1) ^ 1, abort_flag);
        if (w != 1) {
          if (w == 0) tc_fail(err, abort_flag);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * N);
        for (int a = 0; a < S::NKA; ++a) {
          const uint32_t st = L % NST, n = L / NST;
          w = tc_wait(split + st, n & 1, abort_flag);
          if (w != 1) {
            if (w == 0) tc_fail(err, abort_flag);
            go = false;
            break;
          }
          tc_fence_after();
          const uint32_t ah = sb + S::OFF_AHI + st * S::A_BYTES, al = sb + S::OFF_ALO + st * S::A_BYTES;
          const uint32_t bh = sb + a * S::B_SLICE, bl = sb + S::OFF_BLO + a * S::B_SLICE;
#pragma unroll
          for (int kk = 0; kk < kTcKA / 8; ++kk) {
            const uint32_t o = 32u * kk;
            tc_mma(d, tc_desc(ah + o), tc_desc(bh + o), S::IDESC, (a | kk) != 0);
            tc_mma(d, tc_desc(ah + o), tc_desc(bl + o), S::IDESC, 1u);
            tc_mma(d, tc_desc(al + o), tc_desc(bh + o), S::IDESC, 1u);
          }
          tc_commit(empty + st);  // the stage is free once these MMAs are done
          ++L;
        }
        if (go) tc_commit(tfull + b);
      }
      // every MMA issued is done before the tensor memory is freed
      tc_commit(drain);
      mbar_wait(drain, 0, kTcPolls);
    }
  } else if (warp < kTcEpi0) {
    // ---- split: hi in place, lo beside it
    const int sid = threadIdx.x - kTcSplit0 * 32;
    uint32_t L = 0;
    bool go = run;
    for (long long t = blockIdx.x; t < ntiles && go; t += gridDim.x) {
      for (int a = 0; a < S::NKA; ++a) {
        const uint32_t st = L % NST, n = L / NST;
        const int w = tc_warp_wait(full + st, n & 1, abort_flag);
        if (w != 1) {
          if (w == 0 && lane == 0) tc_fail(err, abort_flag);
          go = false;
          break;
        }
        float4 *hi = reinterpret_cast<float4 *>(base + S::OFF_AHI + st * S::A_BYTES);
        float4 *lo = reinterpret_cast<float4 *>(base + S::OFF_ALO + st * S::A_BYTES);
#pragma unroll 4
        for (int i = sid; i < (int)(S::A_BYTES / 16); i += (kTcEpi0 - kTcSplit0) * 32) {
          float4 x = hi[i], l;
          tc_split4(x, l);
          hi[i] = x;
          lo[i] = l;
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(split + st);
        ++L;
      }
    }
  } else {
    // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. of the
    // accumulator (rows), columns [h HC, (h + 1) HC)
    constexpr int HC = N / 2;
    const int q = warp & 3, h = (warp - kTcEpi0) >> 2;
    int it = 0;
    bool go = run;
    for (long long t = blockIdx.x; t < ntiles && go; t += gridDim.x, ++it) {
      const int b = it & 1;
      const uint32_t u = (uint32_t)it >> 1;
      const long long rbase = t * kTcBM + q * 32;  // the warp's first row
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * N + h * HC);
      {
        const int w = tc_warp_wait(tfull + b, u & 1, abort_flag);
        if (w != 1) {
          if (w == 0 && lane == 0) tc_fail(err, abort_flag);
          break;
        }
        tc_fence_after();
        const long long row = rbase + lane;
#pragma unroll 1
        for (int c = 0; c < HC; c += 32) {
          float v[32];
          tc_ld32(taddr + (uint32_t)c, v);
          if (row < rows) {
            float4 *o = reinterpret_cast<float4 *>(out + row * N + h * HC + c);
#pragma unroll
            for (int j = 0; j < 8; ++j) o[j] = make_float4(s * v[4 * j], s * v[4 * j + 1], s * v[4 * j + 2], s * v[4 * j + 3]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty + b);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TCOLS) : "memory");
  }
}

// ---- the prolongation with half rows per CTA and the residual by TMA
//
// out [rows][N] = y [rows][K] P^T - s r.  CTA b computes the column half
// h = b mod 2 of its rows, so it holds only that half of the split table
// (P rows [h NH, (h + 1) NH), NH = N / 2: 64 KB instead of 128 KB for N =
// 256), and the space that frees is a ring of 32-column residual chunks
// ([128 rows][32 floats], 128-byte swizzle) that a producer warp fills by
// TMA ahead of the epilogue; the epilogue writes out = acc - s r in place
// and stores the chunk by TMA.  The row tile of y is read by both CTAs of a
// pair (50 MB more at 256^3, against 400 MB of residual and result that
// now move as whole 128-byte rows with 80 KB in flight per SM).
//
//   warp 0      TMA: the table half once, then the two K slices of y
//   warp 1      MMA issuer (N = NH), tensor-memory allocation
//   warps 2-5   split hi / lo
//   warp 6      TMA: residual chunks into the ring
//   warps 7-10  epilogue, warp w the tensor-memory lanes 32 (w % 4) ..
constexpr int kP2Warps = 11;
constexpr int kP2Threads = kP2Warps * 32;
constexpr int kP2Epi0 = 7;
constexpr int kP2Ring = 5;

template <int K, int N> struct P2Shape {
  static constexpr int NH = N / 2;
  static_assert(K % kTcKA == 0 && NH % 32 == 0 && NH <= 256, "K slices of 32 floats, half rows of 32-column chunks");
  static constexpr int NKA = K / kTcKA;
  static constexpr int NST = NKA;                     // stages: one row tile
  static constexpr int NCH = NH / 32;                 // residual chunks per item
  static constexpr uint32_t A_BYTES = kTcBM * 128;
  static constexpr uint32_t B_SLICE = NH * 128;
  static constexpr uint32_t B_BYTES = NKA * B_SLICE;
  static constexpr uint32_t R_BYTES = kTcBM * 128;    // one residual chunk
  static constexpr uint32_t OFF_BLO = B_BYTES;
  static constexpr uint32_t OFF_AHI = 2 * B_BYTES;
  static constexpr uint32_t OFF_ALO = OFF_AHI + NST * A_BYTES;
  static constexpr uint32_t OFF_RING = OFF_ALO + NST * A_BYTES;
  static constexpr uint32_t OFF_BAR = OFF_RING + kP2Ring * R_BYTES;
  // full, split, empty per stage; tfull[2], tempty[2]; bfull; drain;
  // rfull, rempty per ring slot; then the tensor-memory address and the
  // abort flag
  static constexpr int NBAR = 3 * NST + 6 + 2 * kP2Ring;
  static constexpr uint32_t OFF_MISC = OFF_BAR + NBAR * 8;
  static constexpr uint32_t SMEM = OFF_MISC + 16 + 1024;
  static constexpr uint32_t TCOLS = 2 * NH <= 128 ? 128 : (2 * NH <= 256 ? 256 : 512);
  static constexpr uint32_t IDESC =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NH >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
};

// OR of v over the 128 epilogue threads (named barrier 1): the epilogue
// warps leave their loops together, so none waits at barrier 1 for a warp
// that has gone.
__device__ __forceinline__ bool p2_epi_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, 1, 128, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void p2_epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, const void *src, int c0, int c1) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(c0), "r"(c1)
               : "memory");
}

// tmy: y [rows][K] (box 32 x 128); tmb: P [N][K] (box 32 x NH); tmr / tmo:
// r / out [rows][N] (box 32 x 128); all with the 128-byte swizzle.
template <int K, int N>
__global__ void __launch_bounds__(kP2Threads, 1)
    k_prolong_x_tc2(long long rows, const __grid_constant__ CUtensorMap tmy, const __grid_constant__ CUtensorMap tmb,
                    const __grid_constant__ CUtensorMap tmr, const __grid_constant__ CUtensorMap tmo, float s,
                    int *__restrict__ err) {
  using S = P2Shape<K, N>;
  constexpr int NST = S::NST, NH = S::NH, NCH = S::NCH;
  extern __shared__ unsigned char tc_raw[];
  unsigned char *base = tc_raw + ((1024u - (smem_u32(tc_raw) & 1023u)) & 1023u);
  const uint32_t sb = smem_u32(base);
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + S::OFF_BAR);
  uint64_t *full = bars, *split = bars + NST, *empty = bars + 2 * NST;
  uint64_t *tfull = bars + 3 * NST, *tempty = tfull + 2, *bfull = tempty + 2, *drain = bfull + 1;
  uint64_t *rfull = drain + 1, *rempty = rfull + kP2Ring;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(base + S::OFF_MISC);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(base + S::OFF_MISC + 4);
  unsigned char *ring = base + S::OFF_RING;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ntiles = (rows + kTcBM - 1) / kTcBM;
  const int h = blockIdx.x & 1;
  const long long t0 = blockIdx.x >> 1, tstep = gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int q = 0; q < NST; ++q) {
      mbar_init(full + q, 1);
      mbar_init(split + q, kTcEpi0 - kTcSplit0);
      mbar_init(empty + q, 1);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(tfull + q, 1);
      mbar_init(tempty + q, kP2Warps - kP2Epi0);
    }
    mbar_init(bfull, 1);
    mbar_init(drain, 1);
    for (int q = 0; q < kP2Ring; ++q) {
      mbar_init(rfull + q, 1);
      mbar_init(rempty + q, 1);
    }
    *abort_flag = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(S::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  // this CTA's half of the table, once, split into hi / lo in place
  if (threadIdx.x == 0) {
    mbar_expect_tx(bfull, S::B_BYTES);
#pragma unroll 1
    for (int a = 0; a < S::NKA; ++a) tma_load_2d(base + a * S::B_SLICE, &tmb, bfull, a * kTcKA, h * NH);
  }
  const bool bok = mbar_wait(bfull, 0, kTcPolls);
  if (__syncthreads_or(!bok)) {
    if (threadIdx.x == 0) {
      tc_fail(err, abort_flag);
      mbar_wait(bfull, 0, kTcPolls);
    }
  } else {
    float4 *bh = reinterpret_cast<float4 *>(base), *bl = reinterpret_cast<float4 *>(base + S::OFF_BLO);
    for (int i = threadIdx.x; i < (int)(S::B_BYTES / 16); i += kP2Threads) {
      float4 x = bh[i], lo;
      tc_split4(x, lo);
      bh[i] = x;
      bl[i] = lo;
    }
    fence_proxy_async();
  }
  __syncthreads();
  const bool run = *abort_flag == 0;

  if (warp == 0) {
    // ---- y row tiles, one K slice per stage
    if (lane == 0 && run) {
      uint32_t L = 0;
      bool go = true;
      for (long long t = t0; t < ntiles && go; t += tstep) {
        for (int a = 0; a < S::NKA; ++a) {
          const uint32_t st = L % NST, n = L / NST;
          const int w = tc_wait(empty + st, (n & 1) ^ 1, abort_flag);
          if (w != 1) {
            if (w == 0) tc_fail(err, abort_flag);
            go = false;
            break;
          }
          mbar_expect_tx(full + st, S::A_BYTES);
          tma_load_2d(base + S::OFF_AHI + st * S::A_BYTES, &tmy, full + st, a * kTcKA, (int)(t * kTcBM));
          ++L;
        }
      }
      for (uint32_t st = 0; st < (uint32_t)NST; ++st)
        if (L > st) mbar_wait(full + st, ((L - 1 - st) / NST) & 1, kTcPolls);
    }
  } else if (warp == 1) {
    // ---- MMA issuer
    if (lane == 0 && run) {
      uint32_t L = 0;
      bool go = true;
      int it = 0;
      for (long long t = t0; t < ntiles && go; t += tstep, ++it) {
        const int b = it & 1;
        const uint32_t u = (uint32_t)it >> 1;
        int w = tc_wait(tempty + b, (u & 1) ^ 1, abort_flag);
        if (w != 1) {
          if (w == 0) tc_fail(err, abort_flag);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * NH);
        for (int a = 0; a < S::NKA; ++a) {
          const uint32_t st = L % NST, n = L / NST;
          w = tc_wait(split + st, n & 1, abort_flag);
          if (w != 1) {
            if (w == 0) tc_fail(err, abort_flag);
            go = false;
            break;
          }
          tc_fence_after();
          const uint32_t ah = sb + S::OFF_AHI + st * S::A_BYTES, al = sb + S::OFF_ALO + st * S::A_BYTES;
          const uint32_t bh = sb + a * S::B_SLICE, bl = sb + S::OFF_BLO + a * S::B_SLICE;
#pragma unroll
          for (int kk = 0; kk < kTcKA / 8; ++kk) {
            const uint32_t o = 32u * kk;
            tc_mma(d, tc_desc(ah + o), tc_desc(bh + o), S::IDESC, (a | kk) != 0);
            tc_mma(d, tc_desc(ah + o), tc_desc(bl + o), S::IDESC, 1u);
            tc_mma(d, tc_desc(al + o), tc_desc(bh + o), S::IDESC, 1u);
          }
          tc_commit(empty + st);
          ++L;
        }
        if (go) tc_commit(tfull + b);
      }
      tc_commit(drain);
      mbar_wait(drain, 0, kTcPolls);
    }
  } else if (warp < kTcEpi0) {
    // ---- split
    const int sid = threadIdx.x - kTcSplit0 * 32;
    uint32_t L = 0;
    bool go = run;
    for (long long t = t0; t < ntiles && go; t += tstep) {
      for (int a = 0; a < S::NKA; ++a) {
        const uint32_t st = L % NST, n = L / NST;
        const int w = tc_warp_wait(full + st, n & 1, abort_flag);
        if (w != 1) {
          if (w == 0 && lane == 0) tc_fail(err, abort_flag);
          go = false;
          break;
        }
        float4 *hi = reinterpret_cast<float4 *>(base + S::OFF_AHI + st * S::A_BYTES);
        float4 *lo = reinterpret_cast<float4 *>(base + S::OFF_ALO + st * S::A_BYTES);
#pragma unroll 4
        for (int i = sid; i < (int)(S::A_BYTES / 16); i += (kTcEpi0 - kTcSplit0) * 32) {
          float4 x = hi[i], l;
          tc_split4(x, l);
          hi[i] = x;
          lo[i] = l;
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(split + st);
        ++L;
      }
    }
  } else if (warp < kP2Epi0) {
    // ---- residual chunks into the ring
    if (lane == 0 && run) {
      uint32_t L = 0;
      bool go = true;
      for (long long t = t0; t < ntiles && go; t += tstep) {
        for (int c = 0; c < NCH; ++c) {
          const uint32_t slot = L % kP2Ring, n = L / kP2Ring;
          const int w = tc_wait(rempty + slot, (n & 1) ^ 1, abort_flag);
          if (w != 1) {
            if (w == 0) tc_fail(err, abort_flag);
            go = false;
            break;
          }
          mbar_expect_tx(rfull + slot, S::R_BYTES);
          tma_load_2d(ring + slot * S::R_BYTES, &tmr, rfull + slot, h * NH + 32 * c, (int)(t * kTcBM));
          ++L;
        }
      }
      for (uint32_t slot = 0; slot < (uint32_t)kP2Ring; ++slot)
        if (L > slot) mbar_wait(rfull + slot, ((L - 1 - slot) / kP2Ring) & 1, kTcPolls);
    }
  } else {
    // ---- epilogue: out = acc - s r in place in the ring slot, stored by TMA
    const int q = warp & 3, row = q * 32 + lane;
    const bool leader = warp == kP2Epi0 && lane == 0;  // issues the stores
    uint32_t L = 0;
    int it = 0;
    bool go = run;
    for (long long t = t0; t < ntiles && go; t += tstep, ++it) {
      const int b = it & 1;
      const uint32_t u = (uint32_t)it >> 1;
      int w = lane == 0 ? tc_wait(tfull + b, u & 1, abort_flag) : 0;
      w = __shfl_sync(0xffffffffu, w, 0);
      if (p2_epi_any(w != 1)) {
        if (w == 0 && lane == 0) tc_fail(err, abort_flag);
        go = false;
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * NH);
#pragma unroll 1
      for (int c = 0; c < NCH; ++c) {
        const uint32_t slot = L % kP2Ring, n = L / kP2Ring;
        w = lane == 0 ? tc_wait(rfull + slot, n & 1, abort_flag) : 0;
        w = __shfl_sync(0xffffffffu, w, 0);
        if (p2_epi_any(w != 1)) {
          if (w == 0 && lane == 0) tc_fail(err, abort_flag);
          go = false;
          break;
        }
        float v[32];
        tc_ld32(taddr + (uint32_t)(32 * c), v);
        // the row's eight 16-byte pieces, at piece j ^ (row mod 8) (the swizzle)
        float4 *rp = reinterpret_cast<float4 *>(ring + slot * S::R_BYTES) + row * 8;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int pj = j ^ (row & 7);
          float4 x = rp[pj];
          x.x = v[4 * j] - s * x.x;
          x.y = v[4 * j + 1] - s * x.y;
          x.z = v[4 * j + 2] - s * x.z;
          x.w = v[4 * j + 3] - s * x.w;
          rp[pj] = x;
        }
        fence_proxy_async();  // the chunk, seen by the TMA store
        p2_epi_sync();
        if (leader) {
          tma_store_2d(&tmo, ring + slot * S::R_BYTES, h * NH + 32 * c, (int)(t * kTcBM));
          tma_commit();
          tma_wait_read0();  // the slot may be refilled once the store has read it
          mbar_arrive(rempty + slot);
        }
        ++L;
      }
      if (!go) break;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty + b);
    }
    if (leader) tma_wait0();  // the stores are complete before the CTA leaves
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TCOLS) : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 tc_encode() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// [outer][inner] FP32 rows, box of 32 floats x box_outer rows, 128-byte swizzle.
bool tc_map(CUtensorMap *m, const float *p, long long inner, long long outer, int box_outer) {
  const auto fn = tc_encode();
  if (!fn || (reinterpret_cast<uintptr_t>(p) & 15) != 0) return false;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)inner * sizeof(float)};
  cuuint32_t box[2] = {(cuuint32_t)kTcKA, (cuuint32_t)box_outer};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(p), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int K, int N>
bool tc_launch(long long rows, const float *a, const float *B, float s, float *out, int *err, cudaStream_t st) {
  using S = TcShape<K, N>;
  static_assert(S::SMEM <= 227 * 1024, "tiles exceed the shared memory of a CTA");
  if (rows < 1 || rows > 0x7fffffffLL - kTcBM) return false;
  if ((reinterpret_cast<uintptr_t>(out) & 15) != 0) return false;
  CUtensorMap ma, mb;
  if (!tc_map(&ma, a, K, rows, kTcBM) || !tc_map(&mb, B, K, N, N)) return false;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return false;
  const void *fn = (const void *)k_transfer_x_tc<K, N>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM) != cudaSuccess)
    return false;
  const long long ntiles = (rows + kTcBM - 1) / kTcBM;
  const unsigned grid = (unsigned)std::min<long long>(ntiles, sms);
  k_transfer_x_tc<K, N><<<grid, kTcThreads, S::SMEM, st>>>(rows, ma, mb, s, out, err);
  return cudaGetLastError() == cudaSuccess;
}

template <int K, int N>
bool tc_prolong2(long long rows, const float *y, const float *P, const float *r, float s, float *out, int *err,
                 cudaStream_t st) {
  using S = P2Shape<K, N>;
  static_assert(S::SMEM <= 227 * 1024, "tiles exceed the shared memory of a CTA");
  if (rows < 1 || rows > 0x7fffffffLL - kTcBM) return false;
  CUtensorMap my, mb, mr, mo;
  if (!tc_map(&my, y, K, rows, kTcBM) || !tc_map(&mb, P, K, N, S::NH) || !tc_map(&mr, r, N, rows, kTcBM) ||
      !tc_map(&mo, out, N, rows, kTcBM))
    return false;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 2)
    return false;
  const void *fn = (const void *)k_prolong_x_tc2<K, N>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM) != cudaSuccess)
    return false;
  const long long ntiles = (rows + kTcBM - 1) / kTcBM;
  const unsigned grid = (unsigned)std::min<long long>(2 * ntiles, sms - sms % 2);  // CTA pairs: both halves of a tile
  k_prolong_x_tc2<K, N><<<grid, kP2Threads, S::SMEM, st>>>(rows, my, mb, mr, mo, s, err);
  return cudaGetLastError() == cudaSuccess;
}

}  // namespace

// (fine, coarse) x lengths with a tensor-core transfer: coarse 64 points,
// fine 128, 192 or 256 (the table, split in hi and lo, stays in shared
// memory beside three pipeline stages).
bool tc_x_has(int n0, int nc) { return nc == 64 && (n0 == 128 || n0 == 192 || n0 == 256); }

// out [rows][nc] = s * in [rows][n0] R^T, R [nc][n0].  False: no kernel for
// this pair, or the launch was refused (nothing was written).
bool tc_restrict_x(long long rows, int n0, int nc, const float *in, float s, const float *R, float *out, int *err,
                   cudaStream_t st) {
  if (!tc_x_has(n0, nc)) return false;
  switch (n0) {
    case 128: return tc_launch<128, 64>(rows, in, R, s, out, err, st);
    case 192: return tc_launch<192, 64>(rows, in, R, s, out, err, st);
    case 256: return tc_launch<256, 64>(rows, in, R, s, out, err, st);
    default: return false;
  }
}

// out [rows][n0] = y [rows][nc] P^T - s r, P [n0][nc].
bool tc_prolong_x(long long rows, int n0, int nc, const float *y, const float *P, const float *r, float s, float *out,
                  int *err, cudaStream_t st) {
  if (!tc_x_has(n0, nc)) return false;
  switch (n0) {
    case 128: return tc_prolong2<64, 128>(rows, y, P, r, s, out, err, st);
    case 192: return tc_prolong2<64, 192>(rows, y, P, r, s, out, err, st);
    case 256: return tc_prolong2<64, 256>(rows, y, P, r, s, out, err, st);
    default: return false;
  }
}

}  // namespace rism
