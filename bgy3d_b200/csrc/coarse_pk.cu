// coarse_pk.cu -- instantiations and cooperative launch of the persistent
// coarse GMRES (coarse_pk.cuh) for the cubic coarse grids with
// shape-specialised transforms: (M, N) = (24, 48), (32, 64), (36, 72),
// (48, 96) in the plane form, (64, 128) in the five-phase form.
#include <cstdlib>

#include "coarse_pk.cuh"

namespace rism {

namespace {

struct PkShape {
  const void *fn;
  size_t smem;
  int phases;
};

// The plane form (three phases per step) where its plane tiles fit two CTAs
// per SM (coarse x half rows up to 48); RISM3D_PK_PLANES=0 selects the
// five-phase form everywhere (comparison tests).
template <int M, int N, bool PL> PkShape pk_make() {
  if constexpr (PL) {
    const char *e = std::getenv("RISM3D_PK_PLANES");
    if (!(e && e[0] == '0'))
      return PkShape{(const void *)k_coarse_gmres<M, N, true>, pk_smem<M, N, true>(), pk_phases<true>()};
  }
  return PkShape{(const void *)k_coarse_gmres<M, N, false>, pk_smem<M, N, false>(), pk_phases<false>()};
}

bool pk_shape(int M, int N, PkShape *s) {
  switch (M * 1000 + N) {
#define PK_CASE(MM, NN, PL)      \
  case MM * 1000 + NN:           \
    *s = pk_make<MM, NN, PL>(); \
    return true;
    PK_CASE(24, 48, true) PK_CASE(32, 64, true) PK_CASE(36, 72, true) PK_CASE(48, 96, true) PK_CASE(64, 128, false)
#undef PK_CASE
    default: return false;
  }
}

}  // namespace

// Grid barriers per GMRES step of the kernel that shape (M, N) runs (0: none).
int coarse_pk_phases(int M, int N) {
  PkShape s{};
  return pk_shape(M, N, &s) ? s.phases : 0;
}

// CTAs of the cooperative grid for shape (M, N): min(per_sm, the resident
// CTAs per SM) x SMs; 0 when the shape has no kernel or nothing fits.
int coarse_pk_grid(int M, int N, int per_sm) {
  PkShape s{};
  if (!pk_shape(M, N, &s)) return 0;
  int dev = 0, sms = 0, coop = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
  // opt in always: the static shared memory counts against the default 48 KB
  if (cudaFuncSetAttribute(s.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem) != cudaSuccess)
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
