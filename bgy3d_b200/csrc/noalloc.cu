// noalloc.cu -- the Jacobian product without any device allocation.
//
// Some callers cannot call cudaMalloc: a non-linear solver that invokes the
// Jacobian action from inside a steady-state loop where allocation would
// synchronise the device or is forbidden by the host framework's memory
// policy, or code that owns every device buffer itself and hands the
// library only its inputs and outputs.  rism3d_jacobian_apply_noalloc serves
// them: it computes J dT = (chi - 1) * (d . dT) - dT with the same passes as
// rism3d_jacobian_t1, but keeps its scratch -- the complex work buffer, the
// twiddle and chi tables and the norm partials -- in the file-scope device
// array below, so it allocates nothing.
//
// The array is a fixed kNoallocScratchBytes (32 MiB) on every device that
// loads the library, held until the process exits; a grid whose scratch does
// not fit is rejected with RISM3D_ERR_ARG.  All calls share it: two calls
// whose work overlaps on the GPU (different streams or host threads) race.
// Nothing in it has to start at zero -- each call writes every region before
// reading it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "rism3d.h"

using namespace rism;

namespace rism {
void set_last_error(const std::string &msg);  // rism3d.cu: the message of rism3d_last_error()
}

namespace {

constexpr size_t kNoallocScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Device address of the array, looked up once per device with that device
// current.  In host code the symbol is only a stand-in, never an address.
std::mutex g_mu;
void *g_addr[64] = {nullptr};

// Records a failed CUDA call for rism3d_last_error() and returns the code.
int cuda_fail(const char *what, cudaError_t e) {
  set_last_error(std::string("rism3d_jacobian_apply_noalloc: ") + what + ": " + cudaGetErrorString(e));
  return RISM3D_ERR_CUDA;
}

int setup(int dev, void **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= 64) {
    set_last_error("rism3d_jacobian_apply_noalloc: device ordinal beyond 63");
    return RISM3D_ERR_ARG;
  }
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress of the scratch array", e);
    if (!p) return cuda_fail("cudaGetSymbolAddress of the scratch array", cudaErrorInvalidSymbol);
    // the passes may use more than 48 KB of dynamic shared memory
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return cuda_fail("cudaDeviceGetAttribute", e);
    const void *fns[] = {(const void *)k_xfwd<double, MODE_J>, (const void *)k_xinv<double>,
                         (const void *)k_y<double, false, 16>, (const void *)k_y<double, true, 16>,
                         (const void *)k_y<double, false, 8>,  (const void *)k_y<double, true, 8>,
                         (const void *)k_y<double, false, 4>,  (const void *)k_y<double, true, 4>,
                         (const void *)k_z<double, MODE_J, 16>, (const void *)k_z<double, MODE_J, 8>,
                         (const void *)k_z<double, MODE_J, 4>};
    for (const void *f : fns) {
      cudaFuncAttributes fa{};
      e = cudaFuncGetAttributes(&fa, f);
      if (e != cudaSuccess) return cuda_fail("cudaFuncGetAttributes", e);
      e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
      if (e != cudaSuccess) return cuda_fail("cudaFuncSetAttribute", e);
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return RISM3D_OK;
}

bool is_2a3b_even(int n) {
  if (n < 8 || n > 512 || n % 2) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

AxisPlan plan_of(int n, const void *tw) {
  AxisPlan p{};
  p.n = n;
  int m = n, s = 0;
  while (m % 4 == 0) { p.rad[s++] = 4; m /= 4; }
  while (m % 2 == 0) { p.rad[s++] = 2; m /= 2; }
  while (m % 3 == 0) { p.rad[s++] = 3; m /= 3; }
  p.nst = s;
  p.tw = tw;
  return p;
}

void twiddles(int n, double2 *out) {
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int q = 0; q < n; ++q) {
    const long double a = 2.0L * pi * (long double)q / (long double)n;
    out[q] = make_double2((double)cosl(a), (double)-sinl(a));
  }
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" int rism3d_jacobian_apply_noalloc(const rism3d_problem *pd, int m, const double *chi, const double *d,
                                             const double *dT, double *JdT) {
  if (!pd || !chi || !d || !dT || !JdT || m < 1 || m > kMaxSites || pd->nrad < 4 || !(pd->rmax > 0)) {
    set_last_error("rism3d_jacobian_apply_noalloc: NULL pointer, site count or chi table out of range");
    return RISM3D_ERR_ARG;
  }
  for (int a = 0; a < 3; ++a)
    if (!is_2a3b_even(pd->N[a]) || !(pd->L[a] > 0)) {
      set_last_error("rism3d_jacobian_apply_noalloc: grid sizes must be even 2^a 3^b in 8..512, box edges > 0");
      return RISM3D_ERR_ARG;
    }
  Geo g{};
  g.N0 = pd->N[0]; g.N1 = pd->N[1]; g.N2 = pd->N[2];
  g.M = g.N0 / 2; g.Nh = g.M + 1; g.Nhp = (g.Nh + 1) & ~1; g.m = m;
  g.Nr = (long long)g.N0 * g.N1 * g.N2;
  g.Nc = (long long)g.Nhp * g.N1 * g.N2;
  const double pi = 3.14159265358979323846;
  g.dk0 = 2 * pi / pd->L[0]; g.dk1 = 2 * pi / pd->L[1]; g.dk2 = 2 * pi / pd->L[2];
  const double dkr = pi / pd->rmax;
  const double kmax = std::sqrt(std::pow(g.M * g.dk0, 2) + std::pow(g.N1 / 2 * g.dk1, 2) + std::pow(g.N2 / 2 * g.dk2, 2));
  if ((int)(kmax / dkr) >= pd->nrad) {
    set_last_error("rism3d_jacobian_apply_noalloc: |k| of the grid beyond the chi table");
    return RISM3D_ERR_TABLE;
  }
  // tile shapes of the FP64 runtime-length passes (8 complex per thread)
  int RX = 32, BY = 16, BZ = 16;
  while (RX > 1 && g.M * RX > 8 * 256) RX /= 2;
  while (BY > 4 && g.N1 * BY > 8 * 256) BY /= 2;
  while (BZ > 4 && g.N2 * BZ > 8 * 256) BZ /= 2;
  if (g.N1 * BY > 8 * 256 || g.N2 * BZ > 8 * 256) {
    set_last_error("rism3d_jacobian_apply_noalloc: grid too long along y or z");
    return RISM3D_ERR_ARG;
  }
  const int rows = g.N1 * g.N2;
  const int nblk = ((rows + RX - 1) / RX) * m;
  const int npair = m * (m + 1) / 2;
  // scratch regions, 256-byte aligned
  size_t off = 0;
  const size_t oW = off;   off += up256(sizeof(double2) * (size_t)m * g.Nc);
  const size_t oTx = off;  off += up256(sizeof(double2) * g.M);
  const size_t oTy = off;  off += up256(sizeof(double2) * g.N1);
  const size_t oTz = off;  off += up256(sizeof(double2) * g.N2);
  const size_t oPo = off;  off += up256(sizeof(double2) * g.Nh);
  const size_t oCh = off;  off += up256(sizeof(double2) * (size_t)npair * pd->nrad);
  const size_t oPa = off;  off += up256(sizeof(NormPartial) * (size_t)nblk);
  if (off > kNoallocScratchBytes) {
    set_last_error("rism3d_jacobian_apply_noalloc: the grid needs " + std::to_string(off) +
                   " bytes of scratch, the limit is " + std::to_string(kNoallocScratchBytes));
    return RISM3D_ERR_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  void *base = nullptr;
  int rc = setup(dev, &base);
  if (rc != RISM3D_OK) return rc;
  unsigned char *S = static_cast<unsigned char *>(base);
  double2 *W = reinterpret_cast<double2 *>(S + oW);
  // host-built tables copied in (no allocation on the device side)
  std::vector<double2> h;
  h.resize(g.M);  twiddles(g.M, h.data());
  if ((e = cudaMemcpy(S + oTx, h.data(), sizeof(double2) * g.M, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail("cudaMemcpy", e);
  h.resize(g.N1); twiddles(g.N1, h.data());
  if ((e = cudaMemcpy(S + oTy, h.data(), sizeof(double2) * g.N1, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail("cudaMemcpy", e);
  h.resize(g.N2); twiddles(g.N2, h.data());
  if ((e = cudaMemcpy(S + oTz, h.data(), sizeof(double2) * g.N2, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail("cudaMemcpy", e);
  h.resize(g.N0); twiddles(g.N0, h.data());
  if ((e = cudaMemcpy(S + oPo, h.data(), sizeof(double2) * g.Nh, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail("cudaMemcpy", e);
  // chi - delta as (value, slope) pairs, the interpolation of bgy3d-vec.c:22-46
  const int nrad = pd->nrad;
  std::vector<double2> tab((size_t)npair * nrad);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j <= i; ++j) {
      const double *row = chi + ((size_t)i * m + j) * nrad;
      double2 *dst = tab.data() + (size_t)(i * (i + 1) / 2 + j) * nrad;
      for (int k = 0; k < nrad; ++k) {
        const int ip = (k < nrad - 2) ? k + 1 : k, im = (k > 1) ? k - 1 : k;
        const double dl = (i == j) ? 1.0 : 0.0;
        dst[k] = make_double2(row[k] - dl, ((row[ip] - dl) - (row[im] - dl)) / (ip - im));
      }
    }
  if ((e = cudaMemcpy(S + oCh, tab.data(), sizeof(double2) * tab.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail("cudaMemcpy", e);
  const AxisPlan px = plan_of(g.M, S + oTx), py = plan_of(g.N1, S + oTy), pz = plan_of(g.N2, S + oTz);
  const double2 *post = reinterpret_cast<const double2 *>(S + oPo);
  ZParams<double> zp{};
  zp.chi = reinterpret_cast<const double2 *>(S + oCh);
  zp.stab = nullptr;
  zp.L = nullptr;
  zp.nrad = nrad;
  zp.dkr = dkr;
  const dim3 gx((rows + RX - 1) / RX, m);
  const size_t sx = sizeof(double2) * (size_t)(g.M + RX * g.M);
  const size_t sy = sizeof(double2) * (size_t)(g.N1 + g.N1 * BY);
  const size_t sz = sizeof(double2) * (size_t)(g.N2 + g.N2 * m * BZ);
  k_xfwd<double, MODE_J><<<gx, 256, sx>>>(g, px, RX, dT, d, 1.0, pd->closure, W, post);
  const dim3 gy((g.Nh + BY - 1) / BY, g.N2, m), gz((g.Nh + BZ - 1) / BZ, g.N1);
  if (BY == 16) k_y<double, false, 16><<<gy, 256, sy>>>(g, py, W);
  else if (BY == 8) k_y<double, false, 8><<<gy, 256, sy>>>(g, py, W);
  else k_y<double, false, 4><<<gy, 256, sy>>>(g, py, W);
  if (BZ == 16) k_z<double, MODE_J, 16><<<gz, 256, sz>>>(g, pz, W, zp);
  else if (BZ == 8) k_z<double, MODE_J, 8><<<gz, 256, sz>>>(g, pz, W, zp);
  else k_z<double, MODE_J, 4><<<gz, 256, sz>>>(g, pz, W, zp);
  if (BY == 16) k_y<double, true, 16><<<gy, 256, sy>>>(g, py, W);
  else if (BY == 8) k_y<double, true, 8><<<gy, 256, sy>>>(g, py, W);
  else k_y<double, true, 4><<<gy, 256, sy>>>(g, py, W);
  k_xinv<double><<<gx, 256, sx>>>(g, px, RX, W, dT, JdT, 1.0 / (double)g.Nr, 1.0, post,
                                  reinterpret_cast<NormPartial *>(S + oPa));
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail("kernel launch", e);
  // the calling thread's own default stream (the library is built with
  // per-thread default streams): other threads' work is not waited for
  if ((e = cudaStreamSynchronize(cudaStreamPerThread)) != cudaSuccess) return cuda_fail("cudaStreamSynchronize", e);
  return RISM3D_OK;
}
