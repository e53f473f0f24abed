// twogrid_yz.cu -- the y and z grid transfers of the two-grid preconditioner
// by FFT (sm_100a).
//
// Along one axis the band-limited restriction R (N -> Nc points) and
// prolongation P (Nc -> N) of twogrid.cuh are
//
//   R v = (1/N)  IDFT_Nc( truncate_w( DFT_N v ) ),
//   P c = (1/Nc) IDFT_N ( pad_w     ( DFT_Nc c ) ),
//
// truncate_w keeping the modes |k| < Nc/2 and folding +-Nc/2 into the
// coarse Nyquist mode with weight 1/2 each, pad_w its transpose (the coarse
// Nyquist mode split in halves onto +-Nc/2, zeros elsewhere).  Both are real
// operators, so two adjacent real columns (a, b) -- one float2 in memory --
// go through as the complex column a + ib and come out as Ra + iRb.  A CTA
// loads a [n_in][16] tile of such column pairs (128-byte rows), transforms it
// in shared memory with the compile-time two-step FFT of fft_static.cuh,
// truncates or pads into a second tile, transforms back and stores
// [n_out][16]: one read and one write of each field, where the dense
// per-axis products (k_transfer_axis*) spend 2 n_in n_out flops per column.
#include <cuda_runtime.h>

#include "fft_static.cuh"

namespace rism {

namespace {

// Complex column pairs per tile: 16 (128-byte rows) where both tiles and the
// twiddles fit the default 48 KB of shared memory, else 8.
template <int NI, int NO> __host__ __device__ constexpr int yz_cols() {
  return (NI + NO) * (16 + 1) * 8 <= 48 * 1024 ? 16 : 8;
}

template <int NI, int NO> __host__ __device__ constexpr size_t yz_smem() {
  return sizeof(float2) * ((size_t)(NI + NO) * yz_cols<NI, NO>() + NI + NO);
}

// in [outer][NI][inner] -> out [outer][NO][inner] floats, inner even.
template <int NI, int NO>
__global__ void __launch_bounds__(256) k_transfer_fft(int outer, int inner, const float *__restrict__ in,
                                                      const float2 *__restrict__ twi, const float2 *__restrict__ two,
                                                      float *__restrict__ out) {
  constexpr int B = yz_cols<NI, NO>();
  extern __shared__ __align__(16) unsigned char yz_raw[];
  float2 *X = reinterpret_cast<float2 *>(yz_raw);  // [NI][B]
  float2 *Y = X + NI * B;                            // [NO][B]
  float2 *ti = Y + NO * B;
  float2 *to = ti + NI;
  const int tid = threadIdx.x;
  const int ntile = (inner + 2 * B - 1) / (2 * B);
  const int o = blockIdx.x / ntile;
  const int i0 = (blockIdx.x - o * ntile) * 2 * B;
  for (int q = tid; q < NI; q += 256) ti[q] = twi[q];
  for (int q = tid; q < NO; q += 256) to[q] = two[q];
  const float *src = in + (long long)o * NI * inner + i0;
  for (int e = tid; e < NI * B; e += 256) {
    const int j = e / B, c = e - j * B;
    X[e] = i0 + 2 * c < inner ? *reinterpret_cast<const float2 *>(src + (long long)j * inner + 2 * c)
                              : make_float2(0.f, 0.f);
  }
  __syncthreads();
  // square splits: over 16 columns the 16 x 4 split of 64 points leaves
  // three quarters of the threads idle in its first step
  fft2<NI, B, 256, false, true, LayCol<NI, B>, SplitSq<NI>>(X, ti);
  const float scale = 1.0f / (float)NI;
  for (int e = tid; e < NO * B; e += 256) {
    const int k = e / B, c = e - k * B;
    float2 v = make_float2(0.f, 0.f);
    if (NO < NI) {  // truncate: coarse mode k from the fine spectrum
      if (2 * k < NO) {
        v = X[k * B + c];
      } else if (2 * k == NO) {
        const float2 a = X[k * B + c], b = X[(NI - k) * B + c];
        v = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
      } else {
        v = X[(NI - NO + k) * B + c];
      }
    } else {  // pad: fine mode k from the coarse spectrum
      if (2 * k < NI) {
        v = X[k * B + c];
      } else if (2 * k == NI || 2 * (NO - k) == NI) {
        const float2 a = X[(NI / 2) * B + c];
        v = make_float2(0.5f * a.x, 0.5f * a.y);
      } else if (NO - k < NI / 2) {
        v = X[(NI - NO + k) * B + c];
      }
    }
    Y[e] = make_float2(v.x * scale, v.y * scale);
  }
  __syncthreads();
  fft2<NO, B, 256, true, true, LayCol<NO, B>, SplitSq<NO>>(Y, to);
  float *dst = out + (long long)o * NO * inner + i0;
  for (int e = tid; e < NO * B; e += 256) {
    const int k = e / B, c = e - k * B;
    if (i0 + 2 * c < inner) *reinterpret_cast<float2 *>(dst + (long long)k * inner + 2 * c) = Y[e];
  }
}

template <int NI, int NO>
bool launch_fft(int outer, int inner, const float *in, const float2 *twi, const float2 *two, float *out,
                cudaStream_t st) {
  constexpr int B = yz_cols<NI, NO>();
  constexpr size_t sm = yz_smem<NI, NO>();
  static_assert(sm <= 48 * 1024, "tile exceeds the default shared memory");
  const long long tiles = (long long)outer * ((inner + 2 * B - 1) / (2 * B));
  if (tiles > 0x7fffffffLL) return false;
  k_transfer_fft<NI, NO><<<(unsigned)tiles, 256, sm, st>>>(outer, inner, in, twi, two, out);
  return true;
}

}  // namespace

// (fine, coarse) axis lengths with a kernel in both directions.
#define YZ_PAIRS(X) X(96, 48) X(128, 48) X(128, 64) X(144, 72) X(192, 64) X(192, 96) X(256, 64) X(256, 72) \
                    X(256, 96) X(256, 128) X(512, 96) X(512, 128)

// out [outer][n_out][inner] = transfer of in [outer][n_in][inner] along the
// middle axis (restriction when n_out < n_in); twi / two: the FP32 twiddle
// tables exp(-2 pi i q / n) of lengths n_in / n_out.  False: no kernel for
// this pair, or inner odd.
bool yz_fft_transfer(int outer, int n_in, int n_out, int inner, const float *in, const float2 *twi,
                     const float2 *two, float *out, cudaStream_t st) {
  if (inner % 2 != 0 || outer < 1) return false;
#define YZ_RUN(F, C)                                                                  \
  if (n_in == F && n_out == C) return launch_fft<F, C>(outer, inner, in, twi, two, out, st); \
  if (n_in == C && n_out == F) return launch_fft<C, F>(outer, inner, in, twi, two, out, st);
  YZ_PAIRS(YZ_RUN)
#undef YZ_RUN
  return false;
}

}  // namespace rism
