// coarse_pk.cu -- instantiations and cooperative launch of the persistent
// coarse GMRES (coarse_pk.cuh) for the cubic coarse grids with
// shape-specialised transforms: (M, N) = (24, 48), (32, 64), (36, 72),
// (48, 96), (64, 128).
#include "coarse_pk.cuh"

namespace rism {

namespace {

template <int M, int N> const void *pk_fn() { return (const void *)k_coarse_gmres<M, N>; }

struct PkShape {
  const void *fn;
  size_t smem;
};

bool pk_shape(int M, int N, PkShape *s) {
  switch (M * 1000 + N) {
#define PK_CASE(MM, NN)                        \
  case MM * 1000 + NN:                         \
    *s = PkShape{pk_fn<MM, NN>(), pk_smem<MM, NN>()}; \
    return true;
    PK_CASE(24, 48) PK_CASE(32, 64) PK_CASE(36, 72) PK_CASE(48, 96) PK_CASE(64, 128)
#undef PK_CASE
    default: return false;
  }
}

}  // namespace

// CTAs of the cooperative grid for shape (M, N): min(per_sm, the resident
// CTAs per SM) x SMs; 0 when the shape has no kernel or nothing fits.
int coarse_pk_grid(int M, int N, int per_sm) {
  PkShape s{};
  if (!pk_shape(M, N, &s)) return 0;
  int dev = 0, sms = 0, coop = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
  if (s.smem > 48 * 1024 &&
      cudaFuncSetAttribute(s.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, s.fn, kPkThreads, s.smem) != cudaSuccess || occ < 1)
    return 0;
  return std::min(occ, std::max(1, per_sm)) * sms;
}

// One coarse solve: zero the barrier counter, launch the grid.
cudaError_t coarse_pk_launch(const PkArgs &a, int M, int N, int grid, cudaStream_t st) {
  PkShape s{};
  if (!pk_shape(M, N, &s) || a.k < 1 || a.k > kPkMaxSteps || a.g.m > 3) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  PkArgs copy = a;
  void *args[] = {&copy};
  return cudaLaunchCooperativeKernel(s.fn, dim3((unsigned)grid), dim3(kPkThreads), args, s.smem, st);
}

}  // namespace rism
