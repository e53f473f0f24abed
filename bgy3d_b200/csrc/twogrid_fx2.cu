// twogrid_fx2.cu -- launchers of the x-axis grid transfers that run both
// sides by FFT (k_restrict_fx2 / k_prolong_fx2 of twogrid_fft.cuh), for the
// (fine half row M, coarse half row MC) pairs that the coarse-grid rule of
// the two-grid preconditioner produces on the shape-specialised grids.
// A separate translation unit so that its instantiations compile in
// parallel with rism3d.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "twogrid_fft.cuh"

namespace rism {

namespace {

constexpr int kRX = 16;  // rows per batch, as the table-product kernels

// Rows per batch of the 128-point half rows (the 256^3 grid): 16 or 32
// (RISM3D_FX2_ROWS, read once).
int rows_128() {
  static const int r = [] {
    const char *e = std::getenv("RISM3D_FX2_ROWS");
    return e && std::atoi(e) == 32 ? 32 : 16;
  }();
  return r;
}

// Persistent CTAs: as many as fit at once, at most `work`; also raises the
// kernel's dynamic shared-memory limit when it needs more than 48 KB.
// Returns 0 when the tile does not fit on this device.
unsigned fx2_grid(const void *fn, size_t smem, unsigned work) {
  int dev = 0, sms = 0, optin = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  if (smem + 4096 > (size_t)optin) return 0;
  if (smem > 48 * 1024 && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 256, smem) != cudaSuccess || per < 1) return 0;
  return std::max(1u, std::min((unsigned)per * (unsigned)sms, work));
}

}  // namespace

// The (M, MC) pairs with an instantiation: coarse grids of 48-256 points
// (half rows 24-128) under fine half rows of 32-256.
#define FX2_PAIRS(X)                                                                                  \
  X(32, 24) X(36, 24) X(48, 24) X(64, 24) X(64, 32) X(72, 24) X(72, 32) X(72, 36) X(96, 24) X(96, 32) \
  X(96, 36) X(96, 48) X(128, 32) X(128, 48) X(128, 64) X(256, 64) X(256, 128)

bool fx2_has_pair(int M, int MC) {
#define FX2_HAS(A, B) if (M == A && MC == B) return true;
  FX2_PAIRS(FX2_HAS)
#undef FX2_HAS
  return false;
}

// out[rows][2 MC] = restriction of s * in[rows][2 M].  false: no kernel for
// this pair or its tile does not fit (the caller then uses the table form).
template <typename T>
bool fx2_restrict(int M, int MC, long long rows, const T *in, float s, const float2 *post, const float2 *tw,
                  const float2 *postc, const float2 *twc, float *out, cudaStream_t st) {
  if (M == 128 && rows_128() == 32) {
    const unsigned nb32 = (unsigned)((rows + 31) / 32);
#define FX2_R32(A, B)                                                                                       \
  if (MC == B) {                                                                                            \
    const size_t sm = fx2_smem<A, B, 32>();                                                                 \
    const unsigned g = fx2_grid((const void *)k_restrict_fx2<T, A, B, 32>, sm, nb32);                       \
    if (g == 0) return false;                                                                               \
    k_restrict_fx2<T, A, B, 32><<<g, 256, sm, st>>>(rows, in, s, post, tw, postc, twc, out);                \
    return true;                                                                                            \
  }
    FX2_R32(128, 32) FX2_R32(128, 48) FX2_R32(128, 64)
#undef FX2_R32
  }
  const unsigned nb = (unsigned)((rows + kRX - 1) / kRX);
#define FX2_R(A, B)                                                                                         \
  if (M == A && MC == B) {                                                                                  \
    const size_t sm = fx2_smem<A, B, kRX>();                                                                \
    const unsigned g = fx2_grid((const void *)k_restrict_fx2<T, A, B, kRX>, sm, nb);                        \
    if (g == 0) return false;                                                                               \
    k_restrict_fx2<T, A, B, kRX><<<g, 256, sm, st>>>(rows, in, s, post, tw, postc, twc, out);               \
    return true;                                                                                            \
  }
  FX2_PAIRS(FX2_R)
#undef FX2_R
  return false;
}

// out[rows][2 M] = prolongation of y[rows][2 MC] - s r.
template <typename T>
bool fx2_prolong(int M, int MC, long long rows, const float *y, const float2 *post, const float2 *tw,
                 const float2 *postc, const float2 *twc, const T *r, double s, T *out, cudaStream_t st) {
  if (M == 128 && rows_128() == 32) {
    const unsigned nb32 = (unsigned)((rows + 31) / 32);
#define FX2_P32(A, B)                                                                                       \
  if (MC == B) {                                                                                            \
    const size_t sm = fx2_smem<A, B, 32>();                                                                 \
    const unsigned g = fx2_grid((const void *)k_prolong_fx2<T, T, A, B, 32>, sm, nb32);                     \
    if (g == 0) return false;                                                                               \
    k_prolong_fx2<T, T, A, B, 32><<<g, 256, sm, st>>>(rows, y, post, tw, postc, twc, r, s, out);            \
    return true;                                                                                            \
  }
    FX2_P32(128, 32) FX2_P32(128, 48) FX2_P32(128, 64)
#undef FX2_P32
  }
  const unsigned nb = (unsigned)((rows + kRX - 1) / kRX);
#define FX2_P(A, B)                                                                                         \
  if (M == A && MC == B) {                                                                                  \
    const size_t sm = fx2_smem<A, B, kRX>();                                                                \
    const unsigned g = fx2_grid((const void *)k_prolong_fx2<T, T, A, B, kRX>, sm, nb);                      \
    if (g == 0) return false;                                                                               \
    k_prolong_fx2<T, T, A, B, kRX><<<g, 256, sm, st>>>(rows, y, post, tw, postc, twc, r, s, out);           \
    return true;                                                                                            \
  }
  FX2_PAIRS(FX2_P)
#undef FX2_P
  return false;
}

template bool fx2_restrict<float>(int, int, long long, const float *, float, const float2 *, const float2 *,
                                  const float2 *, const float2 *, float *, cudaStream_t);
template bool fx2_restrict<double>(int, int, long long, const double *, float, const float2 *, const float2 *,
                                   const float2 *, const float2 *, float *, cudaStream_t);
template bool fx2_prolong<float>(int, int, long long, const float *, const float2 *, const float2 *,
                                 const float2 *, const float2 *, const float *, double, float *, cudaStream_t);
template bool fx2_prolong<double>(int, int, long long, const float *, const float2 *, const float2 *,
                                  const float2 *, const float2 *, const double *, double, double *, cudaStream_t);

}  // namespace rism
