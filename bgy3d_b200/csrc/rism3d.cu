// rism3d.cu -- host side of the B200-native 3D-RISM solute solver: the
// C ABI of include/rism3d.h, the device-resident problem context, the
// residual / Jacobian pipelines and the Newton-GMRES driver.
//
// Reference: hnc3d_solute_solve (hnc3d.c:1762-2350) driving iterate_t1 /
// jacobian_t1 (hnc3d.c:1183-1362) through bgy3d_snes_newton
// (bgy3d-snes.c:160-346, SNESNEWTONLS + KSPGMRES(30), KSP rtol = 100 * 1e-5).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <system_error>
#include <thread>
#include <tuple>
#include <vector>

#include "coarse_pk.cuh"
#include "kernels.cuh"
#include "kernels_static.cuh"
#include "grad.cuh"
#include "krylov.cuh"
#include "info.cuh"
#include "rism3d.h"
#include "solvent.cuh"
#include "twogrid.cuh"
#include "twogrid_fft.cuh"

using namespace rism;

namespace rism {  // twogrid_fx2.cu: x transfers with both sides by FFT
bool fx2_has_pair(int M, int MC);
// twogrid_yz.cu: y / z transfers by FFT
bool yz_fft_transfer(int outer, int n_in, int n_out, int inner, const float *in, const float2 *twi,
                     const float2 *two, float *out, cudaStream_t st);
// coarse_pk.cu: the persistent cooperative coarse GMRES
int coarse_pk_grid(int M, int N, int per_sm);
int coarse_pk_phases(int M, int N);
cudaError_t coarse_pk_launch(const PkArgs &a, int M, int N, int grid, cudaStream_t st);
template <typename T>
bool fx2_restrict(int M, int MC, long long rows, const T *in, float s, const float2 *post, const float2 *tw,
                  const float2 *postc, const float2 *twc, float *out, cudaStream_t st);
template <typename T>
bool fx2_prolong(int M, int MC, long long rows, const float *y, const float2 *post, const float2 *tw,
                 const float2 *postc, const float2 *twc, const T *r, double s, T *out, cudaStream_t st);
// twogrid_tc.cu: the x transfers of FP32 data on the tensor cores
bool tc_x_has(int n0, int nc);
bool tc_restrict_x(long long rows, int n0, int nc, const float *in, float s, const float *R, float *out, int *err,
                   cudaStream_t st);
bool tc_prolong_x(long long rows, int n0, int nc, const float *y, const float *P, const float *r, float s, float *out,
                  int *err, cudaStream_t st);
}  // namespace rism

namespace {

thread_local std::string g_last_error;

struct CudaFail {
  int code;
};

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);              \
      throw CudaFail{e_ == cudaErrorMemoryAllocation ? RISM3D_ERR_NOMEM : RISM3D_ERR_CUDA}; \
    }                                                                                 \
  } while (0)

#define CKL()                                                                         \
  do {                                                                                \
    cudaError_t e_ = cudaGetLastError();                                              \
    if (e_ != cudaSuccess) {                                                          \
      g_last_error = std::string("kernel launch: ") + cudaGetErrorString(e_);         \
      throw CudaFail{RISM3D_ERR_CUDA};                                                \
    }                                                                                 \
  } while (0)

struct ArgFail {
  int code;
  std::string msg;
};

// Device memory comes from the device's stream-ordered pool on the calling
// thread's default stream (the library is built with per-thread default
// streams): unlike cudaMalloc / cudaFree it never synchronises the device,
// so solves set up and torn down by concurrent host threads (the batch
// driver) do not stall one another.  The pool keeps freed memory for reuse.
void pool_setup() {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  CK(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t keep = UINT64_MAX;
  CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  done[dev] = true;
}

template <typename T> T *dalloc(size_t count) {
  pool_setup();
  void *p = nullptr;
  if (count == 0) count = 1;
  CK(cudaMallocAsync(&p, count * sizeof(T), cudaStreamPerThread));
  return static_cast<T *>(p);
}

// Stream-ordered free on the calling thread's stream: callers free only
// memory whose last use was on that stream or has completed.
void dfree(void *p) {
  if (p) cudaFreeAsync(p, cudaStreamPerThread);
}

// Pinned landing buffer of the calling host thread for reduced Krylov
// coefficients (4 * 32 doubles), allocated on first use and kept for the
// thread's lifetime: contexts come and go without pinning or unpinning
// host memory, which would synchronise the device.
double *pinned_scratch() {
  struct Buf {
    double *p = nullptr;
    ~Buf() {
      if (p) cudaFreeHost(p);
    }
  };
  static thread_local Buf b;
  if (!b.p) CK(cudaMallocHost(&b.p, sizeof(double) * 4 * kVecMax));
  return b.p;
}

bool is_2a3b(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

AxisPlan make_plan(int n) {
  AxisPlan p{};
  p.n = n;
  int m = n, s = 0;
  while (m % 4 == 0) { p.rad[s++] = 4; m /= 4; }
  while (m % 2 == 0) { p.rad[s++] = 2; m /= 2; }
  while (m % 3 == 0) { p.rad[s++] = 3; m /= 3; }
  p.nst = s;
  return p;
}

// exp(-2 pi i q / n) in extended precision, rounded once.
void twiddles(int n, std::vector<double2> &t64, std::vector<float2> &t32) {
  t64.resize(n);
  t32.resize(n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int q = 0; q < n; ++q) {
    const long double a = 2.0L * pi * (long double)q / (long double)n;
    const long double c = cosl(a), s = -sinl(a);
    t64[q] = make_double2((double)c, (double)s);
    t32[q] = make_float2((float)c, (float)s);
  }
}

// The radial interpolation rule of bgy3d-vec.c:22-46 as (value, slope)
// pairs: f(x) = tab[i] + slope[i] * (x/dx - 1/2 - i), i = nearest entry.
void interp_pairs(const double *tab, int n, std::vector<double2> &out) {
  out.resize(n);
  for (int i = 0; i < n; ++i) {
    const int ip = (i < n - 2) ? i + 1 : i;
    const int im = (i > 0 + 1) ? i - 1 : i;
    const double fi = (tab[ip] - tab[im]) / (ip - im);
    out[i] = make_double2(tab[i], fi);
  }
}

}  // namespace

// ---------------------------------------------------------------- context
// Tile shapes of the passes: RX rows per x-pass CTA, BY / BZ kx-columns per
// y / z-pass CTA; chosen so that n * batch <= reg_complex * 256 threads.
struct TileShape {
  int RX = 16, BY = 8, BZ = 8;
};

struct PassTimer {
  bool on = false;
  cudaEvent_t a, b;
  double ms[12] = {0};
  long long launches[12] = {0};
};

struct rism3d_ctx {
  rism3d_problem pd;
  int m = 0, n = 0;
  Geo g{};
  long long nvec = 0;  // m * Nr
  TileShape tiles[2];  // [0]: FP64 passes, [1]: FP32 passes
  std::vector<rism3d_site> solvent, solute;
  std::vector<double> charge;
  double h3 = 0, dkr = 0;

  AxisPlan px64{}, py64{}, pz64{}, px32{}, py32{}, pz32{};
  double2 *tw64[3] = {nullptr, nullptr, nullptr};
  float2 *tw32[3] = {nullptr, nullptr, nullptr};
  double2 *post64 = nullptr;
  float2 *post32 = nullptr;

  double *v64 = nullptr;
  double *uc64 = nullptr;   // long-range Coulomb field of the solute (observables), or null
  bool uc_valid = false;    // uc64 matches the bound solute
  float *v32 = nullptr;
  double2 *L64 = nullptr;
  float2 *L32 = nullptr;
  double2 *chi64 = nullptr, *s64 = nullptr;
  float2 *chi32 = nullptr, *s32 = nullptr;
  double2 *chi3_64 = nullptr;  // chi - 1 on the k grid (W layout, packed pairs), or null
  float2 *chi3_32 = nullptr;
  // pure-solvent context: solvent sites (0 for a solute context), the pair
  // constants of its OZ z pass and C(k) at the last residual's point
  int pure = 0;
  std::vector<double> pq2, pwr;
  double2 *ck = nullptr;
  void *W = nullptr;  // complex work buffer, FP64-sized, reused by the FP32 path
  SiteP *d_solute = nullptr, *d_solvent = nullptr;
  int n_cap = 0;  // capacity of d_solute
  double *d_charge = nullptr;

  NormPartial *npart = nullptr;
  double *dpart = nullptr;       // [red_blocks][kVecMax] reduction partials
  double *dres = nullptr;        // [kVecMax * 2] reduced coefficients (device)
  std::vector<double> h_dpart;
  int red_blocks = 592;

  // solver work (lazily allocated)
  double *F64 = nullptr, *X64t = nullptr, *F64t = nullptr;
  float *X32 = nullptr, *F32 = nullptr, *X32t = nullptr, *F32t = nullptr;
  double *d64 = nullptr;
  float *d32 = nullptr;
  std::vector<double *> basis64;
  std::vector<float *> basis32;
  double *dx64 = nullptr;
  float *dx32 = nullptr;
  std::vector<double *> zbasis64;  // flexible-GMRES preconditioned directions
  std::vector<float *> zbasis32;

  // two-grid preconditioner: the coarse problem and the per-axis transfer
  // matrices R [Nc][N], Rt [N][Nc], P [N][Nc], Pt [Nc][N] (FP32)
  rism3d_ctx *coarse = nullptr;
  int Nc[3] = {0, 0, 0};
  float *tR[3] = {nullptr, nullptr, nullptr}, *tRt[3] = {nullptr, nullptr, nullptr};
  float *tP[3] = {nullptr, nullptr, nullptr}, *tPt[3] = {nullptr, nullptr, nullptr};
  float2 *tC = nullptr, *tD = nullptr;     // x-axis FFT-transfer tables
  float *tA = nullptr, *tB = nullptr;       // partially transferred fields
  float *tc_r = nullptr, *tc_y = nullptr;   // coarse right-hand side / solution
  int coarse_jv = 0;
  // the coarse solve as one CUDA graph (device-driven GMRES, no host syncs)
  cudaGraph_t cg_graph = nullptr;
  cudaGraphExec_t cg_exec = nullptr;
  double *cg_H = nullptr, *cg_aux = nullptr;  // Hessenberg columns; norm, beta, y
  unsigned *cg_ticket = nullptr;              // last-block ticket of the fused sweeps
  long long cg_nodes = 0;
  bool cg_failed = false;
  // the coarse solve as one persistent cooperative kernel (coarse_pk.cuh)
  double *pk_dot = nullptr, *pk_nrm = nullptr;  // block partials of its reductions
  unsigned *pk_bar = nullptr;                   // its grid-barrier counter
  int pk_grid = 0;                              // CTAs (0: not set up)
  bool pk_failed = false;                       // shape or device without it
  int coarse_driver = -1;  // of the last coarse solve: 0 host-driven, 1 graph, 2 persistent kernel
  double2 *phase_tab = nullptr;  // per-axis phase factors of the solute form factor [3 axes][phase_cap][n_a]
  int phase_cap = 0;
  unsigned long long *pk_trace = nullptr;       // RISM3D_PK_TRACE: phase timestamps
  unsigned long long *pk_trace_cta = nullptr;   // RISM3D_PK_TRACE=3: every CTA at every barrier

  cudaStream_t stream = 0;
  PassTimer timer;
  int f_evals = 0, jv_evals = 0, f32_evals = 0, jv32_evals = 0;

  // shape-specialised passes: available per precision ([0] FP64, [1] FP32),
  // with TMA descriptors of W for the y and z tiles
  bool stat[2] = {false, false};
  int zb[2] = {4, 8};  // z tile width of the shape-specialised z pass ([0] FP64, [1] FP32: 8 or 4)
  bool zpers[2] = {false, false};  // that z pass from persistent double-buffered CTAs
  CUtensorMap tmy[2], tmz[2];
  int *d_err = nullptr;  // set by a kernel whose bounded wait timed out

  ~rism3d_ctx() {
    auto fr = [](void *p) { dfree(p); };
    for (int i = 0; i < 3; ++i) { fr(tw64[i]); fr(tw32[i]); }
    fr(post64); fr(post32); fr(v64); fr(uc64); fr(v32); fr(L64); fr(L32);
    fr(chi64); fr(s64); fr(chi32); fr(s32); fr(chi3_64); fr(chi3_32); fr(ck); fr(W); fr(d_solute); fr(d_solvent); fr(d_charge);
    fr(npart); fr(dpart); fr(dres); fr(F64); fr(X64t); fr(F64t); fr(X32); fr(F32); fr(X32t); fr(F32t);
    fr(d64); fr(d32); fr(dx64); fr(dx32); fr(d_err);
    for (auto p : basis64) fr(p);
    for (auto p : basis32) fr(p);
    for (auto p : zbasis64) fr(p);
    for (auto p : zbasis32) fr(p);
    for (int a = 0; a < 3; ++a) { fr(tR[a]); fr(tRt[a]); fr(tP[a]); fr(tPt[a]); }
    fr(tA); fr(tB); fr(tc_r); fr(tc_y); fr(cg_H); fr(cg_aux); fr(cg_ticket); fr(tC); fr(tD);
    fr(pk_dot); fr(pk_nrm); fr(pk_bar); fr(pk_trace); fr(pk_trace_cta); fr(phase_tab);
    if (cg_exec) cudaGraphExecDestroy(cg_exec);
    if (cg_graph) cudaGraphDestroy(cg_graph);
    delete coarse;
    if (timer.on) { cudaEventDestroy(timer.a); cudaEventDestroy(timer.b); }
  }

  template <typename T> const AxisPlan &plan(int axis) const;
  template <typename T> typename Cx<T>::type *work() { return static_cast<typename Cx<T>::type *>(W); }
  template <typename T> const TileShape &tl() const { return tiles[sizeof(T) == 8 ? 0 : 1]; }
};

template <> const AxisPlan &rism3d_ctx::plan<double>(int a) const { return a == 0 ? px64 : (a == 1 ? py64 : pz64); }
template <> const AxisPlan &rism3d_ctx::plan<float>(int a) const { return a == 0 ? px32 : (a == 1 ? py32 : pz32); }

namespace {

enum { TK_XFWD = 0, TK_Y = 1, TK_Z = 2, TK_XINV = 3, TK_VEC = 4, TK_PREC = 5 };

// Times one pass (when enabled) into bucket which + 6 * precision and
// always counts its kernel launches.
struct TimeScope {
  rism3d_ctx *c;
  int which;
  TimeScope(rism3d_ctx *c_, int w, int prec, int nlaunch = 1) : c(c_), which(w + 6 * prec) {
    c->timer.launches[which] += nlaunch;
    if (c->timer.on) cudaEventRecord(c->timer.a, c->stream);
  }
  ~TimeScope() {
    if (c->timer.on) {
      cudaEventRecord(c->timer.b, c->stream);
      cudaEventSynchronize(c->timer.b);
      float ms = 0;
      cudaEventElapsedTime(&ms, c->timer.a, c->timer.b);
      c->timer.ms[which] += ms;
    }
  }
};

template <typename T> ZParams<T> zparams(rism3d_ctx *c, bool full);
template <> ZParams<double> zparams<double>(rism3d_ctx *c, bool full) {
  ZParams<double> z{};
  z.chi = c->chi64;
  z.chi3 = c->chi3_64;
  z.stab = (full && c->pd.renorm) ? c->s64 : nullptr;
  z.L = full ? c->L64 : nullptr;
  z.nrad = c->pd.nrad;
  z.dkr = c->dkr;
  for (int i = 0; i < c->m && !c->pure; ++i) {
    z.a[i] = c->pd.renorm ? 0.0 : c->pd.beta * c->charge[i];
    z.bconst[i] = c->pd.renorm ? 0.0 : c->pd.beta * c->charge[i];
  }
  return z;
}
template <> ZParams<float> zparams<float>(rism3d_ctx *c, bool full) {
  ZParams<float> z{};
  z.chi = c->chi32;
  z.chi3 = c->chi3_32;
  z.stab = (full && c->pd.renorm) ? c->s32 : nullptr;
  z.L = full ? c->L32 : nullptr;
  z.nrad = c->pd.nrad;
  z.dkr = c->dkr;
  for (int i = 0; i < c->m && !c->pure; ++i) {
    z.a[i] = c->pd.renorm ? 0.f : (float)(c->pd.beta * c->charge[i]);
    z.bconst[i] = c->pd.renorm ? 0.f : (float)(c->pd.beta * c->charge[i]);
  }
  return z;
}

template <typename T> const T *vfield(rism3d_ctx *c);
template <> const double *vfield<double>(rism3d_ctx *c) { return c->v64; }
template <> const float *vfield<float>(rism3d_ctx *c) { return c->v32; }
template <typename T> const typename Cx<T>::type *postw(rism3d_ctx *c);
template <> const double2 *postw<double>(rism3d_ctx *c) { return c->post64; }
template <> const float2 *postw<float>(rism3d_ctx *c) { return c->post32; }

template <typename T> size_t xsmem(rism3d_ctx *c) {
  return sizeof(typename Cx<T>::type) * (size_t)(c->g.M + c->tl<T>().RX * c->g.M);
}
template <typename T> size_t ysmem(rism3d_ctx *c) {
  return sizeof(typename Cx<T>::type) * (size_t)(c->g.N1 + c->g.N1 * c->tl<T>().BY);
}
template <typename T> size_t zsmem(rism3d_ctx *c) {
  return sizeof(typename Cx<T>::type) * (size_t)(c->g.N2 + c->g.N2 * c->m * c->tl<T>().BZ);
}

// ---- shape-specialised passes
constexpr int kStaticRX = 16;
// y tile width: 128-byte rows (16 float2 or 8 double2); z tile width: 64-byte
// rows, so the m-site z tile is half as large and four CTAs share an SM
template <typename T> constexpr int static_B() { return sizeof(T) == 4 ? 16 : 8; }
template <typename T> constexpr int static_Bz() { return sizeof(T) == 4 ? 8 : 4; }
template <typename T, int M> constexpr size_t xs_smem() {
  return sizeof(typename Cx<T>::type) * (size_t)(M + kStaticRX * LayRow<M, SplitRow<M>::R2>::RS);
}
template <typename T, int N> constexpr size_t ys_smem() {
  return sizeof(typename Cx<T>::type) * (size_t)(N * static_B<T>() + N) + 16;
}
template <typename T, int N> size_t zs_smem(int m, int B = static_Bz<T>()) {
  return sizeof(typename Cx<T>::type) * (size_t)(m * N * B + N) + 16;
}
template <typename T, int N> size_t zsp_smem(int m) {  // two tile buffers, two mbarriers
  return sizeof(typename Cx<T>::type) * (size_t)(2 * m * N * static_Bz<T>() + N) + 16;
}
// Lengths with shape-specialised passes: the coarse grids (48, 96) and the
// even 2^a 3^b grids of the many-solute workloads whose two-step split fits
// the register transforms (108 and 162 do not: no split of 54 / odd 81).
bool static_len_x(int M) {
  return M == 24 || M == 32 || M == 36 || M == 48 || M == 64 || M == 72 || M == 96 || M == 128 || M == 256;
}
bool static_len_yz(int N) {
  return N == 48 || N == 64 || N == 72 || N == 96 || N == 128 || N == 144 || N == 192 || N == 256 || N == 512;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {  // thread-safe one-time lookup
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  if (!fn) {
    g_last_error = "cuTensorMapEncodeTiled unavailable";
    throw CudaFail{RISM3D_ERR_CUDA};
  }
  return fn;
}

// W viewed as a 3D tensor of scalars {2 Nhp, N1, m N2}; box {2B, by, bz}.
void make_tmap(rism3d_ctx *c, CUtensorMap *tm, bool fp64, int B, int by, int bz) {
  const Geo &G = c->g;
  const size_t es = fp64 ? 8 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)(2 * G.Nhp), (cuuint64_t)G.N1, (cuuint64_t)G.N2 * G.m};
  cuuint64_t strides[2] = {(cuuint64_t)(2 * G.Nhp) * es, (cuuint64_t)(2 * G.Nhp) * G.N1 * es};
  // a box spans at most 256 elements per dimension (the kernels move
  // 512-point tiles as two boxes)
  cuuint32_t box[3] = {(cuuint32_t)(2 * B), (cuuint32_t)std::min(by, 256), (cuuint32_t)std::min(bz, 256)};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode_fn()(tm, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                                 c->W, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    g_last_error = "cuTensorMapEncodeTiled failed: " + std::to_string((int)r);
    throw CudaFail{RISM3D_ERR_CUDA};
  }
}

template <typename T, bool INV> void launch_y(rism3d_ctx *c) {
  TimeScope ts(c, TK_Y, sizeof(T) == 8 ? 0 : 1);
  auto *W = c->work<T>();
  if (c->stat[sizeof(T) == 8 ? 0 : 1]) {
    constexpr int B = static_B<T>();
    dim3 grid((c->g.Nh + B - 1) / B, c->g.N2, c->m);
    const CUtensorMap &tm = c->tmy[sizeof(T) == 8 ? 0 : 1];
    const auto *tw = static_cast<const typename Cx<T>::type *>(c->plan<T>(1).tw);
    switch (c->g.N1) {
#define Y_CASE(N)                                                                                   \
  case N:                                                                                           \
    k_y_s<T, INV, N, B><<<grid, Split<N>::R1 * B, ys_smem<T, N>(), c->stream>>>(c->g, tm, tw, c->d_err); \
    break;
      Y_CASE(48) Y_CASE(64) Y_CASE(72) Y_CASE(96) Y_CASE(128) Y_CASE(144) Y_CASE(192) Y_CASE(256) Y_CASE(512)
#undef Y_CASE
    }
    CKL();
    return;
  }
  dim3 grid((c->g.Nh + c->tl<T>().BY - 1) / c->tl<T>().BY, c->g.N2, c->m);
  const size_t sm = ysmem<T>(c);
  if (c->tl<T>().BY == 16) k_y<T, INV, 16><<<grid, 256, sm, c->stream>>>(c->g, c->plan<T>(1), W);
  else if (c->tl<T>().BY == 8) k_y<T, INV, 8><<<grid, 256, sm, c->stream>>>(c->g, c->plan<T>(1), W);
  else k_y<T, INV, 4><<<grid, 256, sm, c->stream>>>(c->g, c->plan<T>(1), W);
  CKL();
}

void allow_smem(const void *fn, size_t need);
unsigned persistent_grid(const void *fn, size_t smem, unsigned work, int threads);
int optin_limit();

// z pass of a pure-solvent context (solvent.cuh), FP64, for MS solvent sites.
template <int MODE, int MS> void launch_oz_ms(rism3d_ctx *c) {
  PureParams<MS> pp{};
  pp.rho = c->pd.rho;
  pp.beta = c->pd.beta;
  pp.h3 = c->h3;
  pp.ck = c->ck;
  for (int p = 0; p < PureParams<MS>::NP; ++p) {
    pp.q2[p] = c->pq2[p];
    pp.wr[p] = c->pwr[p];
  }
  const int B = c->tl<double>().BZ;
  dim3 grid((c->g.Nh + B - 1) / B, c->g.N1);
  const size_t sm = zsmem<double>(c);
  auto *W = c->work<double>();
  if (B == 16) k_z_oz<MODE, 16, MS><<<grid, 256, sm, c->stream>>>(c->g, c->plan<double>(2), W, pp);
  else if (B == 8) k_z_oz<MODE, 8, MS><<<grid, 256, sm, c->stream>>>(c->g, c->plan<double>(2), W, pp);
  else k_z_oz<MODE, 4, MS><<<grid, 256, sm, c->stream>>>(c->g, c->plan<double>(2), W, pp);
  CKL();
}
template <int MODE> void launch_oz(rism3d_ctx *c) {
  switch (c->pure) {
    case 1: launch_oz_ms<MODE, 1>(c); break;
    case 2: launch_oz_ms<MODE, 2>(c); break;
    case 3: launch_oz_ms<MODE, 3>(c); break;
    default: launch_oz_ms<MODE, 4>(c); break;
  }
}
template <int MODE, int MS> void allow_oz_ms(size_t need) {
  allow_smem((const void *)k_z_oz<MODE, 16, MS>, need);
  allow_smem((const void *)k_z_oz<MODE, 8, MS>, need);
  allow_smem((const void *)k_z_oz<MODE, 4, MS>, need);
}
template <int MS> void allow_oz(size_t need) {
  allow_oz_ms<MODE_F, MS>(need);
  allow_oz_ms<MODE_J, MS>(need);
  allow_oz_ms<MODE_VL, MS>(need);
}

template <typename T, int MODE> void launch_z(rism3d_ctx *c) {
  TimeScope ts(c, TK_Z, sizeof(T) == 8 ? 0 : 1);
  if (c->pure) {
    if constexpr (sizeof(T) == 8 && (MODE == MODE_F || MODE == MODE_J)) {
      launch_oz<MODE>(c);
      return;
    }
    g_last_error = "pure-solvent passes are FP64 residual and Jacobian only";
    throw ArgFail{RISM3D_ERR_UNSUPPORTED, g_last_error};
  }
  auto *W = c->work<T>();
  const ZParams<T> zp = zparams<T>(c, MODE == MODE_F);
  if (c->stat[sizeof(T) == 8 ? 0 : 1]) {
    constexpr int BW = static_Bz<T>(), BN = static_Bz<T>() / 2;  // wide / narrow tiles
    const int B = c->zb[sizeof(T) == 8 ? 0 : 1];
    dim3 grid((c->g.Nh + B - 1) / B, c->g.N1);
    const CUtensorMap &tm = c->tmz[sizeof(T) == 8 ? 0 : 1];
    const auto *tw = static_cast<const typename Cx<T>::type *>(c->plan<T>(2).tw);
    switch (c->g.N2) {
#define Z_CASE(N)                                                                                          \
  case N:                                                                                                  \
    if (B == BW && c->zpers[sizeof(T) == 8 ? 0 : 1]) {                                                     \
      const unsigned nt = (unsigned)(((c->g.Nh + BW - 1) / BW) * c->g.N1);                                 \
      const size_t sm = zsp_smem<T, N>(c->m);                                                               \
      const void *fn = (const void *)k_z_sp<T, MODE, N, BW, 3>;                                             \
      k_z_sp<T, MODE, N, BW, 3><<<persistent_grid(fn, sm, nt, Split<N>::R1 * BW), Split<N>::R1 * BW, sm,    \
                                  c->stream>>>(c->g, tm, tw, zp, c->d_err);                                \
    } else if (B == BW)                                                                                    \
      k_z_s<T, MODE, N, BW, 3><<<grid, Split<N>::R1 * BW, zs_smem<T, N>(c->m, BW), c->stream>>>(c->g, tm, tw, \
                                                                                               zp, c->d_err); \
    else                                                                                                   \
      k_z_s<T, MODE, N, BN, 3><<<grid, Split<N>::R1 * BN, zs_smem<T, N>(c->m, BN), c->stream>>>(c->g, tm, tw, \
                                                                                               zp, c->d_err); \
    break;
      Z_CASE(48) Z_CASE(64) Z_CASE(72) Z_CASE(96) Z_CASE(128) Z_CASE(144) Z_CASE(192) Z_CASE(256) Z_CASE(512)
#undef Z_CASE
    }
    CKL();
    return;
  }
  dim3 grid((c->g.Nh + c->tl<T>().BZ - 1) / c->tl<T>().BZ, c->g.N1);
  const size_t sm = zsmem<T>(c);
  if (c->tl<T>().BZ == 16) k_z<T, MODE, 16><<<grid, 256, sm, c->stream>>>(c->g, c->plan<T>(2), W, zp);
  else if (c->tl<T>().BZ == 8) k_z<T, MODE, 8><<<grid, 256, sm, c->stream>>>(c->g, c->plan<T>(2), W, zp);
  else k_z<T, MODE, 4><<<grid, 256, sm, c->stream>>>(c->g, c->plan<T>(2), W, zp);
  CKL();
}

void reduce_norms(rism3d_ctx *c, int nblk, double *resid) {
  double *dout = c->dres + 2 * kVecMax;
  k_norm_final<<<1, 1024, 0, c->stream>>>(nblk, c->npart, c->d_err, dout);
  CKL();
  double *h = pinned_scratch();
  CK(cudaMemcpyAsync(h, dout, sizeof(double) * 3, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int err = (int)h[2];
  if (err) {
    g_last_error = err == kPkErr   ? std::string("a bounded grid-barrier wait timed out in the coarse solve")
                   : err == kTcErr ? std::string("a bounded mbarrier wait timed out in a tensor-core grid transfer")
                                   : "a bounded TMA/mbarrier wait timed out in pass " + std::to_string(err);
    throw CudaFail{RISM3D_ERR_CUDA};
  }
  resid[0] = h[0];
  resid[1] = std::sqrt(h[1]);
}

// The five passes of one residual (MODE_F: A = t, Bv = v, p = beta) or
// Jacobian product (MODE_J: A = dt, Bv = d = c'(t), p = scale of dt);
// out = (FFT^-1 ...) / N - sub * A.  Returns the number of norm partials.
template <typename T, int MODE>
int pipeline(rism3d_ctx *c, const T *A, const T *Bv, T p, T sub, T *out) {
  const int rows = c->g.N1 * c->g.N2;
  auto *W = c->work<T>();
  const bool st = c->stat[sizeof(T) == 8 ? 0 : 1];
  const int RX = st ? kStaticRX : c->tl<T>().RX;
  dim3 gx((rows + RX - 1) / RX, c->m);
  const auto *twx = static_cast<const typename Cx<T>::type *>(c->plan<T>(0).tw);
  {
    TimeScope ts(c, TK_XFWD, sizeof(T) == 8 ? 0 : 1);
    if (st) {
      switch (c->g.M) {
#define XF_CASE(M)                                                                                     \
  case M:                                                                                              \
    k_xfwd_s<T, MODE, M, kStaticRX><<<gx, 256, xs_smem<T, M>(), c->stream>>>(c->g, A, Bv, p, c->pd.closure, \
                                                                             W, postw<T>(c), twx);      \
    break;
        XF_CASE(24) XF_CASE(32) XF_CASE(36) XF_CASE(48) XF_CASE(64) XF_CASE(72) XF_CASE(96) XF_CASE(128)
        XF_CASE(256)
#undef XF_CASE
      }
    } else {
      k_xfwd<T, MODE><<<gx, 256, xsmem<T>(c), c->stream>>>(c->g, c->plan<T>(0), RX, A, Bv, p, c->pd.closure, W,
                                                          postw<T>(c));
    }
    CKL();
  }
  launch_y<T, false>(c);
  launch_z<T, MODE>(c);
  launch_y<T, true>(c);
  {
    TimeScope ts(c, TK_XINV, sizeof(T) == 8 ? 0 : 1);
    const T scale = (T)(1.0 / (double)c->g.Nr);
    if (st) {
      switch (c->g.M) {
#define XI_CASE(M)                                                                                            \
  case M:                                                                                                     \
    k_xinv_s<T, M, kStaticRX><<<gx, 256, xs_smem<T, M>(), c->stream>>>(c->g, W, A, out, scale, sub, postw<T>(c), \
                                                                       twx, c->npart);                        \
    break;
        XI_CASE(24) XI_CASE(32) XI_CASE(36) XI_CASE(48) XI_CASE(64) XI_CASE(72) XI_CASE(96) XI_CASE(128)
        XI_CASE(256)
#undef XI_CASE
      }
    } else {
      k_xinv<T><<<gx, 256, xsmem<T>(c), c->stream>>>(c->g, c->plan<T>(0), RX, W, A, out, scale, sub, postw<T>(c),
                                                     c->npart);
    }
    CKL();
  }
  return gx.x * gx.y;
}

// F(x) -> out (iterate_t1).  resid: ||out||_inf, ||out||_2 (host), or null.
template <typename T> void eval_F(rism3d_ctx *c, const T *x, T *out, double *resid) {
  const int nb = pipeline<T, MODE_F>(c, x, vfield<T>(c), (T)c->pd.beta, (T)1, out);
  if (sizeof(T) == 8) c->f_evals++; else c->f32_evals++;
  if (resid) reduce_norms(c, nb, resid);
}

// out = J(x0) (s * vin) with d = c'(x0) precomputed (jacobian_t1).
template <typename T> void eval_J(rism3d_ctx *c, const T *d, const T *vin, double s, T *out, double *resid) {
  const int nb = pipeline<T, MODE_J>(c, vin, d, (T)s, (T)s, out);
  if (sizeof(T) == 8) c->jv_evals++; else c->jv32_evals++;
  if (resid) reduce_norms(c, nb, resid);
}

int vec_grid(long long n) {
  long long b = (n + 255) / 256;
  return (int)std::min<long long>(b, 148LL * 8);
}

template <typename T> VecRef<T> vref(const T *p, double s) { return VecRef<T>{p, s}; }

// h[i] = <w * ws, s_i V_i> for i < nv: one sweep per kVecMax basis vectors,
// partials summed on the device.
template <typename T>
void mdot(rism3d_ctx *c, const T *w, double ws, const std::vector<VecRef<T>> &V, std::vector<double> &h) {
  const int nv = (int)V.size();
  const int chunks = (nv + kVecMax - 1) / kVecMax;
  TimeScope ts(c, TK_VEC, sizeof(T) == 8 ? 0 : 1, 2 * chunks);
  h.assign(nv, 0.0);
  const int G = c->red_blocks;
  const long long nw = c->nvec / Wide<T>::n;
  for (int base = 0; base < nv; base += kVecMax) {
    const int k = std::min(kVecMax, nv - base);
    VecSet<T> vs{};
    for (int i = 0; i < kVecMax; ++i) vs.p[i] = V[base + (i < k ? i : 0)].p;
    launch_mdotv<T>(G, c->stream, nw, w, k, vs, c->dpart);
    CKL();
    k_colsum<<<1, kColsumThreads, 0, c->stream>>>(G, kVecMax, k, c->dpart, c->dres + base);
    CKL();
  }
  double *hres = pinned_scratch();
  CK(cudaMemcpyAsync(hres, c->dres, sizeof(double) * nv, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < nv; ++i) h[i] = hres[i] * ws * V[i].s;
}

// w = ws * w - sum_i coef_i (s_i V_i); returns ||w||_2 if want_norm.
template <typename T>
double maxpy(rism3d_ctx *c, T *w, double ws, const std::vector<VecRef<T>> &V, const std::vector<double> &coef,
             bool want_norm) {
  const int nv = (int)V.size();
  const int chunks = std::max(1, (nv + kVecMax - 1) / kVecMax);
  TimeScope ts(c, TK_VEC, sizeof(T) == 8 ? 0 : 1, chunks + (want_norm ? 1 : 0));
  const int G = c->red_blocks;
  const long long nw = c->nvec / Wide<T>::n;
  for (int base = 0; base < std::max(nv, 1); base += kVecMax) {
    const int k = std::min(kVecMax, nv - base);
    VecSet<T> vs{};
    Coefs cf{};
    for (int i = 0; i < kVecMax; ++i) {
      vs.p[i] = i < k ? V[base + i].p : w;
      cf.c[i] = i < k ? coef[base + i] * V[base + i].s : 0.0;
    }
    const bool last = base + kVecMax >= nv;
    launch_maxpyv<T>(G, c->stream, nw, w, base == 0 ? ws : 1.0, std::max(k, 0), vs, cf, nullptr,
                     (last && want_norm) ? c->dpart : nullptr);
    CKL();
  }
  if (!want_norm) return 0.0;
  k_colsum<<<1, kColsumThreads, 0, c->stream>>>(G, 1, 1, c->dpart, c->dres);
  CKL();
  double *hres = pinned_scratch();
  CK(cudaMemcpyAsync(hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return std::sqrt(hres[0]);
}

// One classical Gram-Schmidt step of w against s_i V_i (nv <= kVecMax) with
// a single host round trip: the dots <w, V_i> stay on the device (dres) and
// feed the update w -= sum_i (s_i^2 <w, V_i>) V_i as device coefficients;
// the dots and |w|^2 come back together.  h_i = s_i <w, V_i>; returns |w|
// after the update.
template <typename T>
double gs_step(rism3d_ctx *c, T *w, const std::vector<VecRef<T>> &V, std::vector<double> &h) {
  const int nv = (int)V.size();
  TimeScope ts(c, TK_VEC, sizeof(T) == 8 ? 0 : 1, 4);
  const int G = c->red_blocks;
  const long long nw = c->nvec / Wide<T>::n;
  VecSet<T> vs{};
  Coefs cf{};
  for (int i = 0; i < kVecMax; ++i) {
    vs.p[i] = V[i < nv ? i : 0].p;
    cf.c[i] = i < nv ? V[i].s * V[i].s : 0.0;
  }
  launch_mdotv<T>(G, c->stream, nw, w, nv, vs, c->dpart);
  CKL();
  k_colsum<<<1, kColsumThreads, 0, c->stream>>>(G, kVecMax, nv, c->dpart, c->dres);
  CKL();
  launch_maxpyv<T>(G, c->stream, nw, w, 1.0, nv, vs, cf, c->dres, c->dpart);
  CKL();
  k_colsum<<<1, kColsumThreads, 0, c->stream>>>(G, 1, 1, c->dpart, c->dres + kVecMax);
  CKL();
  double *hres = pinned_scratch();
  CK(cudaMemcpyAsync(hres, c->dres, sizeof(double) * (kVecMax + 1), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  h.assign(nv, 0.0);
  for (int i = 0; i < nv; ++i) h[i] = hres[i] * V[i].s;
  return std::sqrt(std::max(hres[kVecMax], 0.0));
}

template <typename TX, typename TY> void axpby(rism3d_ctx *c, double a, const TX *x, double b, TY *y) {
  TimeScope ts(c, TK_VEC, sizeof(TY) == 8 ? 0 : 1);
  k_axpby<TX, TY><<<vec_grid(c->nvec), 256, 0, c->stream>>>(c->nvec, a, x, b, y);
  CKL();
}
template <typename TX, typename TY, typename TZ>
void xpay(rism3d_ctx *c, const TX *x, double a, const TY *y, TZ *z) {
  TimeScope ts(c, TK_VEC, sizeof(TZ) == 8 ? 0 : 1);
  k_xpay<TX, TY, TZ><<<vec_grid(c->nvec), 256, 0, c->stream>>>(c->nvec, x, a, y, z);
  CKL();
}

template <typename T> std::vector<T *> &basis(rism3d_ctx *c);
template <> std::vector<double *> &basis<double>(rism3d_ctx *c) { return c->basis64; }
template <> std::vector<float *> &basis<float>(rism3d_ctx *c) { return c->basis32; }

template <typename T> void ensure_basis(rism3d_ctx *c, int count) {
  auto &B = basis<T>(c);
  while ((int)B.size() < count) B.push_back(dalloc<T>(c->nvec));
}

// GMRES(restart) without preconditioner for J x = b, x0 = 0 (KSPGMRES with
// classical Gram-Schmidt, PCNONE; bgy3d-snes.c:262-306).  Returns the
// number of J.v products.  b is only read: the first cycle's basis starts
// from b in place.
template <typename T>
int gmres(rism3d_ctx *c, const T *d, const T *b, T *x, double rtol, int maxit, int restart) {
  ensure_basis<T>(c, restart + 1);
  auto &B = basis<T>(c);
  std::vector<double> H((size_t)(restart + 1) * restart), cs(restart), sn(restart), gv(restart + 1);
  std::vector<VecRef<T>> V;
  std::vector<double> h;
  int its = 0;
  bool have_x = false;
  double beta0 = -1.0;
  while (its < maxit) {
    // r = b - J x (first cycle: r = b)
    // r0 = b in the first cycle (read in place: the norm-only sweep writes
    // nothing), else B0 = b - J x
    T *r0 = const_cast<T *>(b);
    if (have_x) {
      eval_J<T>(c, d, x, 1.0, B[0], nullptr);  // B0 = J x
      xpay<T, T, T>(c, b, -1.0, B[0], B[0]);   // B0 = b - J x
      r0 = B[0];
      its++;
    }
    const double beta = maxpy<T>(c, r0, 1.0, {}, {}, true);
    if (beta0 < 0) beta0 = beta;
    if (beta == 0.0 || beta <= rtol * beta0) break;
    V.assign(1, vref<T>(r0, 1.0 / beta));
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    int j = 0;
    bool done = false;
    for (; j < restart && its < maxit; ++j) {
      eval_J<T>(c, d, V[j].p, V[j].s, B[j + 1], nullptr);
      its++;
      double hn;
      if ((int)V.size() <= kVecMax) {
        hn = gs_step<T>(c, B[j + 1], V, h);
      } else {
        mdot<T>(c, B[j + 1], 1.0, V, h);
        hn = maxpy<T>(c, B[j + 1], 1.0, V, h, true);
      }
      for (int i = 0; i <= j; ++i) H[(size_t)i * restart + j] = h[i];
      H[(size_t)(j + 1) * restart + j] = hn;
      for (int i = 0; i < j; ++i) {  // previous Givens rotations
        const double a = H[(size_t)i * restart + j], bb = H[(size_t)(i + 1) * restart + j];
        H[(size_t)i * restart + j] = cs[i] * a + sn[i] * bb;
        H[(size_t)(i + 1) * restart + j] = -sn[i] * a + cs[i] * bb;
      }
      const double a = H[(size_t)j * restart + j], bb = H[(size_t)(j + 1) * restart + j];
      const double r = std::hypot(a, bb);
      cs[j] = r == 0.0 ? 1.0 : a / r;
      sn[j] = r == 0.0 ? 0.0 : bb / r;
      H[(size_t)j * restart + j] = r;
      H[(size_t)(j + 1) * restart + j] = 0.0;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      V.push_back(vref<T>(B[j + 1], hn > 0.0 ? 1.0 / hn : 0.0));
      if (std::fabs(gv[j + 1]) <= rtol * beta0 || hn == 0.0) { ++j; done = true; break; }
    }
    // y = H^-1 g, x += sum y_i V_i
    const int k = j;
    std::vector<double> y(k);
    for (int i = k - 1; i >= 0; --i) {
      double s = gv[i];
      for (int l = i + 1; l < k; ++l) s -= H[(size_t)i * restart + l] * y[l];
      y[i] = H[(size_t)i * restart + i] != 0.0 ? s / H[(size_t)i * restart + i] : 0.0;
    }
    std::vector<VecRef<T>> Vk(V.begin(), V.begin() + k);
    std::vector<double> my(k);
    for (int i = 0; i < k; ++i) my[i] = -y[i];
    maxpy<T>(c, x, have_x ? 1.0 : 0.0, Vk, my, false);
    have_x = true;
    if (done) break;
  }
  if (!have_x) axpby<T, T>(c, 0.0, b, 0.0, x);
  return its;
}

template <typename T> T *xbuf(rism3d_ctx *c, int which);
template <> double *xbuf<double>(rism3d_ctx *c, int w) {
  double **p = w == 0 ? &c->F64 : (w == 1 ? &c->X64t : &c->F64t);
  if (!*p) *p = dalloc<double>(c->nvec);
  return *p;
}
template <> float *xbuf<float>(rism3d_ctx *c, int w) {
  float **p = w == 0 ? &c->F32 : (w == 1 ? &c->X32t : &c->F32t);
  if (!*p) *p = dalloc<float>(c->nvec);
  return *p;
}
template <typename T> T *slopebuf(rism3d_ctx *c);
template <> double *slopebuf<double>(rism3d_ctx *c) { if (!c->d64) c->d64 = dalloc<double>(c->nvec); return c->d64; }
template <> float *slopebuf<float>(rism3d_ctx *c) { if (!c->d32) c->d32 = dalloc<float>(c->nvec); return c->d32; }
template <typename T> T *dxbuf(rism3d_ctx *c);
template <> double *dxbuf<double>(rism3d_ctx *c) { if (!c->dx64) c->dx64 = dalloc<double>(c->nvec); return c->dx64; }
template <> float *dxbuf<float>(rism3d_ctx *c) { if (!c->dx32) c->dx32 = dalloc<float>(c->nvec); return c->dx32; }

template <typename TS> __global__ void k_slope_any(long long n, const TS *__restrict__ t, const double *__restrict__ v,
                                                   double beta, int closure, float *__restrict__ d32,
                                                   double *__restrict__ d64) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double d = closure_d<double>(closure, beta * v[p], (double)t[p]);
  if (d32) d32[p] = (float)d;
  if (d64) d64[p] = d;
}

// The FP32 Jacobian's slope from an FP32 state: FP32 arithmetic on the
// FP32 potential (the one the FP32 residual passes use), four elements per
// thread; the FP64 potential and FP64 exponentials were most of
// k_slope_any's time and are lost in the FP32 result anyway.
__global__ void k_slope_f32(long long n, const float *__restrict__ t, const float *__restrict__ v, float beta,
                            int closure, float *__restrict__ d) {
  const long long n4 = n / 4;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (long long)gridDim.x * blockDim.x) {
    const float4 tv = reinterpret_cast<const float4 *>(t)[q], vv = reinterpret_cast<const float4 *>(v)[q];
    float4 o;
    o.x = closure_d<float>(closure, beta * vv.x, tv.x);
    o.y = closure_d<float>(closure, beta * vv.y, tv.y);
    o.z = closure_d<float>(closure, beta * vv.z, tv.z);
    o.w = closure_d<float>(closure, beta * vv.w, tv.w);
    reinterpret_cast<float4 *>(d)[q] = o;
  }
  if (blockIdx.x == 0 && threadIdx.x < (unsigned)(n - 4 * n4)) {
    const long long p = 4 * n4 + threadIdx.x;
    d[p] = closure_d<float>(closure, beta * v[p], t[p]);
  }
}

template <typename TS, typename TJ> void closure_slope(rism3d_ctx *c, const TS *x, TJ *d) {
  TimeScope ts(c, TK_VEC, sizeof(TJ) == 8 ? 0 : 1);
  const long long n = c->nvec;
  if constexpr (sizeof(TS) == 4 && sizeof(TJ) == 4) {
    if (c->v32 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 && (reinterpret_cast<uintptr_t>(d) & 15) == 0) {
      k_slope_f32<<<vec_grid(n / 4 + 1), 256, 0, c->stream>>>(n, x, c->v32, (float)c->pd.beta, c->pd.closure, d);
      CKL();
      return;
    }
  }
  float *d32 = sizeof(TJ) == 4 ? reinterpret_cast<float *>(d) : nullptr;
  double *d64 = sizeof(TJ) == 8 ? reinterpret_cast<double *>(d) : nullptr;
  k_slope_any<TS><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, x, c->v64, c->pd.beta, c->pd.closure,
                                                                       d32, d64);
  CKL();
}

// ------------------------------------------------ two-grid preconditioner
// M^-1 v = P (J_H^-1 + I) R v - v.  The slow modes of J = (chi-1)*(c' .) - 1
// are long-wavelength fields confined to the solute core, where c' -> -1
// and J -> -chi, whose charge branch vanishes as k -> 0; a coarse problem
// on the same box at about 1 A spacing resolves them, and everywhere else
// (c' = 0, or wavelengths the coarse grid does not hold) J is close to -1.
// R and P are the band-limited transfers of twogrid.cuh.  J_H takes its
// slope from the fine one, c'_H = R c': exp(-beta v + R t) on the coarse
// points would overshoot the fine slope many times over in the attractive
// shells of an unconverged HNC state and wreck the preconditioner there.
// J_H^-1 is a fixed number of FP32 GMRES steps on the coarse context, so M
// varies slightly from call to call and the outer solver is flexible GMRES.

long long launch_total(const rism3d_ctx *c) {
  long long s = 0;
  for (long long l : c->timer.launches) s += l;
  return s;
}

// The y (axis 1) or z (axis 2) transfer of [outer][n_in][inner] into
// [outer][n_out][inner]: by FFT (twogrid_yz.cu) where that pair of lengths
// has a kernel, else as the dense product with A (RISM3D_DENSE_TRANSFERS=1
// forces the dense form, for the comparison tests).  Slab width J of the
// dense form: 32 outputs per thread for the restrictions (n_out <= 64: the
// input is read at most twice), 16 for the prolongations, 8 where the
// threads of a narrow slab would not fill the GPU.
void transfer_axis(rism3d_ctx *c, int axis, int outer, int n_in, int n_out, int inner, const float *in,
                   const float *A, float *out) {
  const char *dense = std::getenv("RISM3D_DENSE_TRANSFERS");
  if (!(dense && dense[0] == '1')) {
    const float2 *tw_fine = c->tw32[axis], *tw_coarse = c->coarse->tw32[axis];
    const bool restrict_ = n_out < n_in;
    if (rism::yz_fft_transfer(outer, n_in, n_out, inner, in, restrict_ ? tw_fine : tw_coarse,
                              restrict_ ? tw_coarse : tw_fine, out, c->stream)) {
      CKL();
      return;
    }
  }
  const long long tot = (long long)outer * inner;
  const unsigned gx = (unsigned)((tot + tg::kAxThreads - 1) / tg::kAxThreads);
  int J = n_out <= 64 ? 32 : 16;
  while (J > 8 && (long long)gx * ((n_out + J - 1) / J) < 2 * 148) J /= 2;
  if (J == 8 || n_in > tg::kAxMaxIn) {
    dim3 g(gx, (unsigned)((n_out + tg::kAxJ - 1) / tg::kAxJ));
    tg::k_transfer_axis<<<g, tg::kAxThreads, 0, c->stream>>>(outer, n_in, n_out, inner, in, A, out);
  } else {
    dim3 g(gx, (unsigned)((n_out + J - 1) / J));
    const size_t sm = sizeof(float) * (size_t)n_in * J;
    if (J == 32) tg::k_transfer_axis_j<32><<<g, tg::kAxThreads, sm, c->stream>>>(outer, n_in, n_out, inner, in, A, out);
    else tg::k_transfer_axis_j<16><<<g, tg::kAxThreads, sm, c->stream>>>(outer, n_in, n_out, inner, in, A, out);
  }
  CKL();
}

// CTAs of a persistent kernel: as many as fit on the device at once
// (`threads` per CTA, `smem` dynamic bytes), at most `work` (the items to walk).
unsigned persistent_grid(const void *fn, size_t smem, unsigned work, int threads) {
  int dev = 0, sms = 0, per = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem));
  const unsigned n = (unsigned)std::max(1, per) * (unsigned)std::max(1, sms);
  return std::max(1u, std::min(n, work));
}

// x-axis transfers by FFT (twogrid_fft.cuh) where the row length has a
// shape-specialised transform; false: use the dense tiles.
constexpr int kFxRX = 16;
bool fx_usable(const rism3d_ctx *c) {
  const char *dense = std::getenv("RISM3D_DENSE_TRANSFERS");  // 1: the dense tiles everywhere (tests)
  if (dense && dense[0] == '1') return false;
  return c->tC && static_len_x(c->g.M) && c->Nc[0] % 2 == 0 && c->Nc[0] / 2 < c->g.M;
}
// Both sides by FFT (twogrid_fx2.cu) where the coarse half row also has a
// shape-specialised transform; RISM3D_DENSE_TRANSFERS=2 keeps the (K+1) x Nc
// table product on the coarse side (tests compare the two).
bool fx2_usable(const rism3d_ctx *c) {
  const char *dense = std::getenv("RISM3D_DENSE_TRANSFERS");
  if (dense && dense[0] == '2') return false;
  return c->coarse && c->coarse->g.M == c->Nc[0] / 2 && rism::fx2_has_pair(c->g.M, c->Nc[0] / 2);
}
template <typename T> bool fx_restrict(rism3d_ctx *c, long long rows, const T *in, double s) {
  if (!fx_usable(c)) return false;
  const int K = c->Nc[0] / 2;
  const auto *post = postw<float>(c);
  const auto *tw = static_cast<const float2 *>(c->plan<float>(0).tw);
  if (fx2_usable(c) && rism::fx2_restrict<T>(c->g.M, c->Nc[0] / 2, rows, in, (float)s, post, tw, c->coarse->post32,
                                              c->coarse->tw32[0], c->tA, c->stream)) {
    CKL();
    return true;
  }
  const unsigned nb = (unsigned)((rows + kFxRX - 1) / kFxRX);
  switch (c->g.M) {
#define FXR(M)                                                                                                 \
  case M: {                                                                                                    \
    const size_t sm = fx_smem_restrict<M, kFxRX>(K, c->Nc[0]);                                                \
    if ((long long)sm > optin_limit()) return false;                                                          \
    if (sm > 48 * 1024) allow_smem((const void *)k_restrict_fx<T, M, kFxRX>, sm);                             \
    k_restrict_fx<T, M, kFxRX><<<persistent_grid((const void *)k_restrict_fx<T, M, kFxRX>, sm, nb, 256), 256, sm,     \
                                 c->stream>>>(rows, c->Nc[0], K, in, (float)s, post, tw, c->tC, c->tA);           \
    break;                                                                                                     \
  }
    FXR(24) FXR(32) FXR(36) FXR(48) FXR(64) FXR(72) FXR(96) FXR(128) FXR(256)
#undef FXR
    default: return false;
  }
  CKL();
  return true;
}
template <typename T> bool fx_prolong(rism3d_ctx *c, long long rows, const T *r, double s, T *out) {
  if (!fx_usable(c)) return false;
  const int K = c->Nc[0] / 2;
  const auto *post = postw<float>(c);
  const auto *tw = static_cast<const float2 *>(c->plan<float>(0).tw);
  if (fx2_usable(c) && rism::fx2_prolong<T>(c->g.M, c->Nc[0] / 2, rows, c->tA, post, tw, c->coarse->post32,
                                             c->coarse->tw32[0], r, s, out, c->stream)) {
    CKL();
    return true;
  }
  const unsigned nb = (unsigned)((rows + kFxRX - 1) / kFxRX);
  switch (c->g.M) {
#define FXP(M)                                                                                                 \
  case M: {                                                                                                    \
    const size_t sm = fx_smem_prolong<M, kFxRX>(K, c->Nc[0]);                                                  \
    if ((long long)sm > optin_limit()) return false;                                                          \
    if (sm > 48 * 1024) allow_smem((const void *)k_prolong_fx<T, T, M, kFxRX>, sm);                           \
    k_prolong_fx<T, T, M, kFxRX><<<persistent_grid((const void *)k_prolong_fx<T, T, M, kFxRX>, sm, nb, 256), 256, sm,  \
                                   c->stream>>>(rows, c->Nc[0], K, c->tA, post, tw, c->tD, r, s, out);            \
    break;                                                                                                     \
  }
    FXP(24) FXP(32) FXP(36) FXP(48) FXP(64) FXP(72) FXP(96) FXP(128) FXP(256)
#undef FXP
    default: return false;
  }
  CKL();
  return true;
}

// The x transfers of FP32 data on the tensor cores (twogrid_tc.cu) where the
// (fine, coarse) pair has a kernel; RISM3D_TC_TRANSFERS=0, or either dense
// switch (RISM3D_DENSE_TRANSFERS=1/2), selects the FFT or dense forms.
bool tc_usable(const rism3d_ctx *c) {
  const char *off = std::getenv("RISM3D_TC_TRANSFERS");
  const char *dense = std::getenv("RISM3D_DENSE_TRANSFERS");
  if ((off && off[0] == '0') || (dense && (dense[0] == '1' || dense[0] == '2'))) return false;
  return c->coarse && c->tR[0] && c->tP[0] && rism::tc_x_has(c->g.N0, c->Nc[0]);
}

// out (coarse [m][Nc2][Nc1][Nc0]) = R (s in), in fine [m][N2][N1][N0].
template <typename T> void tg_restrict(rism3d_ctx *c, const T *in, double s, float *out) {
  const Geo &G = c->g;
  const long long rows = (long long)c->m * G.N2 * G.N1;
  bool tc = false;
  if constexpr (sizeof(T) == 4) {
    if (tc_usable(c)) {
      tc = rism::tc_restrict_x(rows, G.N0, c->Nc[0], in, (float)s, c->tR[0], c->tA, c->d_err, c->stream);
      CKL();
    }
  }
  if (!tc && !fx_restrict<T>(c, rows, in, s)) {
    dim3 gx((unsigned)((rows + tg::kRxRows - 1) / tg::kRxRows),
            (unsigned)((c->Nc[0] + tg::kRxCols - 1) / tg::kRxCols));
    tg::k_restrict_x<T><<<gx, tg::kRxThreads, 0, c->stream>>>(rows, G.N0, c->Nc[0], in, (float)s, c->tRt[0], c->tA);
    CKL();
  }
  transfer_axis(c, 1, c->m * G.N2, G.N1, c->Nc[1], c->Nc[0], c->tA, c->tR[1], c->tB);
  transfer_axis(c, 2, c->m, G.N2, c->Nc[2], c->Nc[1] * c->Nc[0], c->tB, c->tR[2], out);
}

// out = P yc - s r (fine), yc coarse.
template <typename T> void tg_prolong(rism3d_ctx *c, const float *yc, const T *r, double s, T *out) {
  const Geo &G = c->g;
  transfer_axis(c, 2, c->m, c->Nc[2], G.N2, c->Nc[1] * c->Nc[0], yc, c->tP[2], c->tB);
  transfer_axis(c, 1, c->m * G.N2, c->Nc[1], G.N1, c->Nc[0], c->tB, c->tP[1], c->tA);
  const long long rows = (long long)c->m * G.N2 * G.N1;
  bool tc = false;
  if constexpr (sizeof(T) == 4) {
    if (tc_usable(c)) {
      tc = rism::tc_prolong_x(rows, G.N0, c->Nc[0], c->tA, c->tP[0], r, (float)s, out, c->d_err, c->stream);
      CKL();
    }
  }
  if (!tc && !fx_prolong<T>(c, rows, r, s, out)) {
    dim3 gx((unsigned)((rows + tg::kPxRows - 1) / tg::kPxRows), (unsigned)((G.N0 + tg::kPxCols - 1) / tg::kPxCols));
    tg::k_prolong_x<T, T><<<gx, tg::kPxThreads, 0, c->stream>>>(rows, G.N0, c->Nc[0], c->tA, c->tPt[0], r, s, out);
    CKL();
  }
}

// Coarse Jacobian of the current Newton step: c'_H = R d, d = c'(t) fine.
template <typename T> void tg_prepare(rism3d_ctx *c, const T *d) {
  TimeScope ts(c, TK_PREC, sizeof(T) == 8 ? 0 : 1, 3);
  tg_restrict<T>(c, d, 1.0, slopebuf<float>(c->coarse));
}

int coarse_steps(const rism3d_ctx *c) {
  return c->pd.coarse_steps > 0 ? std::min(c->pd.coarse_steps, kVecMax - 1) : 16;
}

// The coarse solve driven entirely on the device: k GMRES steps from zero
// on J_H with an explicitly normalised basis, the dot products and norms
// reduced into device memory, the small least-squares problem solved by one
// thread, and tc_y = sum y_j V_j = J_H^-1 r + r written at the end.  On
// entry the coarse basis vector 0 holds r; nothing here waits for the host,
// so the whole sequence is captured once as a CUDA graph.
void coarse_solve_dev(rism3d_ctx *c, int k) {
  rism3d_ctx *cc = c->coarse;
  auto &B = basis<float>(cc);
  const float *d = cc->d32;
  const int G = cc->red_blocks;
  const long long nw = cc->nvec / Wide<float>::n;
  const int gv = vec_grid(cc->nvec);
  cudaStream_t st = cc->stream;
  double *H = c->cg_H, *nrm = c->cg_aux, *beta = c->cg_aux + 1, *y = c->cg_aux + 2;
  Coefs one{}, mone{};
  for (int i = 0; i < kVecMax; ++i) one.c[i] = 1.0, mone.c[i] = -1.0;
  launch_maxpyv<float>(G, st, nw, B[0], 1.0, 0, VecSet<float>{}, one, nullptr, cc->dpart);
  k_colsum<<<1, kColsumThreads, 0, st>>>(G, 1, 1, cc->dpart, nrm);  // |r|^2
  k_scale_norm<float><<<gv, 256, 0, st>>>(cc->nvec, B[0], nrm, beta);
  CKL();
  for (int j = 0; j < k; ++j) {
    pipeline<float, MODE_J>(cc, B[j], d, 1.f, 1.f, B[j + 1]);
    VecSet<float> vs{};
    for (int i = 0; i < kVecMax; ++i) vs.p[i] = B[i <= j ? i : 0];
    double *h = H + (size_t)j * (k + 1);
    // classical Gram-Schmidt, each sweep with its reduction fused in
    launch_mdot_red<float>(G, st, nw, B[j + 1], j + 1, vs, cc->dpart, c->cg_ticket, h);
    k_maxpy_red<float><<<G, 256, 0, st>>>(nw, B[j + 1], j + 1, vs, h, cc->dpart, c->cg_ticket, h + j + 1);
    k_scale_by<float><<<gv, 256, 0, st>>>(cc->nvec, B[j + 1], h + j + 1);
    CKL();
  }
  k_arnoldi_lsq<<<1, 1, 0, st>>>(k, H, beta, y);
  VecSet<float> vs{};
  for (int i = 0; i < kVecMax; ++i) vs.p[i] = B[i < k ? i : 0];
  launch_maxpyv<float>(G, st, nw, c->tc_y, 0.0, k, vs, mone, y, nullptr);
  CKL();
}

// Capture coarse_solve_dev once (on a private stream; it is launched into the
// context's stream afterwards).  False, with the host-driven path left to
// the caller, when capture or instantiation fails.
bool coarse_graph(rism3d_ctx *c, int k) {
  if (c->cg_exec) return true;
  if (c->cg_failed) return false;
  const char *env = std::getenv("RISM3D_COARSE_GRAPH");  // 0: host-driven coarse GMRES
  if (env && env[0] == '0') {
    c->cg_failed = true;
    return false;
  }
  rism3d_ctx *cc = c->coarse;
  ensure_basis<float>(cc, k + 1);  // every buffer the graph touches exists before capture
  slopebuf<float>(cc);
  if (!c->cg_H) c->cg_H = dalloc<double>((size_t)k * (k + 1));
  if (!c->cg_aux) c->cg_aux = dalloc<double>((size_t)k + 2);
  if (!c->cg_ticket) {
    c->cg_ticket = dalloc<unsigned>(1);
    CK(cudaMemsetAsync(c->cg_ticket, 0, sizeof(unsigned), c->stream));
  }
  cudaStream_t cap = nullptr;
  CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaStream_t saved = cc->stream;
  cc->stream = cap;
  cudaGraph_t g = nullptr;
  bool ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    try {
      coarse_solve_dev(c, k);
    } catch (const CudaFail &) {
      ok = false;
    }
    if (cudaStreamEndCapture(cap, &g) != cudaSuccess) ok = false;
  }
  cc->stream = saved;
  cudaStreamDestroy(cap);
  if (ok && g) {
    size_t n = 0;
    ok = cudaGraphGetNodes(g, nullptr, &n) == cudaSuccess &&
         cudaGraphInstantiate(&c->cg_exec, g, 0) == cudaSuccess;
    c->cg_nodes = (long long)n;
  }
  if (ok) {
    c->cg_graph = g;
  } else {
    if (g) cudaGraphDestroy(g);
    c->cg_exec = nullptr;
    c->cg_failed = true;
    cudaGetLastError();  // capture errors are not sticky; clear the record
  }
  return ok;
}

// Solves issued by concurrent host threads (the batch driver) take the
// graph-replayed coarse solve.  RISM3D_PK_BATCH=1 gives them the persistent
// kernel, serialised on the device (below: cooperative grids of several
// streams could each hold part of the GPU while waiting for the rest).
// Measured on the 64-solute batch: launches 304 k -> 46 k, but 26.6 -> 21.4
// solves/s, since one whole-GPU grid at a time stops the streams' coarse
// solves from overlapping; hence off by default.
thread_local bool tl_concurrent_solves = false;

bool pk_in_batch() {
  static const bool on = [] {
    const char *e = std::getenv("RISM3D_PK_BATCH");
    return e && e[0] == '1';
  }();
  return on;
}

// One cooperative grid at a time on a device: each persistent launch from a
// concurrent solve waits (on the device, not the host) for the previous
// one's completion event, then records its own into the same event.
struct PkSerial {
  std::mutex mu;
  std::map<int, cudaEvent_t> last;  // per device, never destroyed
};
PkSerial &pk_serial() {
  static PkSerial *s = new PkSerial;  // outlives every context
  return *s;
}

// The persistent coarse GMRES is used when the coarse grid is a cube with
// shape-specialised transforms, m <= 3 and k <= 16 (RISM3D_COARSE_PERSIST=0
// turns it off); its buffers are allocated on first use.
bool coarse_pk_ready(rism3d_ctx *c, int k) {
  const bool allowed = !tl_concurrent_solves || pk_in_batch();
  if (c->pk_grid > 0) return allowed;
  if (c->pk_failed || !allowed) return false;
  const char *env = std::getenv("RISM3D_COARSE_PERSIST");
  rism3d_ctx *cc = c->coarse;
  const Geo &G = cc->g;
  if ((env && env[0] == '0') || !cc->stat[1] || cc->pure || G.m > 3 || k < 1 || k > kPkMaxSteps ||
      G.N0 != G.N1 || G.N1 != G.N2) {
    c->pk_failed = true;
    return false;
  }
  const char *per = std::getenv("RISM3D_PK_CTAS_PER_SM");  // CTAs per SM (default 2)
  const int grid = coarse_pk_grid(G.M, G.N1, per ? std::atoi(per) : 2);
  if (grid <= 0) {
    c->pk_failed = true;
    cudaGetLastError();
    return false;
  }
  ensure_basis<float>(cc, k + 1);
  slopebuf<float>(cc);
  c->pk_dot = dalloc<double>((size_t)grid * kVecMax);
  c->pk_nrm = dalloc<double>((size_t)2 * grid);
  c->pk_bar = dalloc<unsigned>(1);
  if (!c->cg_H) c->cg_H = dalloc<double>((size_t)k * (k + 1));
  if (!c->cg_aux) c->cg_aux = dalloc<double>((size_t)k + 2);
  c->pk_grid = grid;
  return true;
}

// J_H^-1 r + r into tc_y by the persistent kernel, r in coarse basis slot 0.
// False (and the kernel off for this context) if the launch is refused.
bool coarse_pk_run(rism3d_ctx *c, int k) {
  rism3d_ctx *cc = c->coarse;
  auto &B = basis<float>(cc);
  PkArgs a{};
  a.g = cc->g;
  a.W = cc->work<float>();
  for (int i = 0; i <= k; ++i) a.V[i] = B[i];
  a.d = slopebuf<float>(cc);
  a.out = c->tc_y;
  a.post = postw<float>(cc);
  a.twx = static_cast<const float2 *>(cc->plan<float>(0).tw);
  a.twy = static_cast<const float2 *>(cc->plan<float>(1).tw);
  a.twz = static_cast<const float2 *>(cc->plan<float>(2).tw);
  a.zp = zparams<float>(cc, false);
  a.pdot = c->pk_dot;
  a.pnrm = c->pk_nrm;
  a.H = c->cg_H;
  a.aux = c->cg_aux;
  a.bar = c->pk_bar;
  a.err = c->d_err;  // read back by the next fine residual's norm check
  a.k = k;
  // RISM3D_PK_TRACE=1: time every phase (synchronises; diagnostics only)
  static const int trace_level = [] {
    const char *t = std::getenv("RISM3D_PK_TRACE");
    return t ? std::atoi(t) : 0;
  }();
  const bool trace = trace_level > 0, trace_steps = trace_level > 1;
  const int P = coarse_pk_phases(cc->g.M, cc->g.N1);  // grid barriers per step
  const int nts = P * k + 4;
  if (trace && !c->pk_trace) c->pk_trace = dalloc<unsigned long long>((size_t)nts);
  a.trace = trace ? c->pk_trace : nullptr;
  const int nbar = P * k + 2;
  const bool trace_ctas = trace_level > 2;
  if (trace_ctas && !c->pk_trace_cta)
    c->pk_trace_cta = dalloc<unsigned long long>((size_t)nbar * 2 * c->pk_grid);
  a.trace_cta = trace_ctas ? c->pk_trace_cta : nullptr;
  cudaError_t e;
  if (tl_concurrent_solves) {
    PkSerial &ps = pk_serial();
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(ps.mu);
    cudaEvent_t &ev = ps.last[dev];
    if (!ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    else CK(cudaStreamWaitEvent(c->stream, ev, 0));
    e = coarse_pk_launch(a, cc->g.M, cc->g.N1, c->pk_grid, c->stream);
    if (e == cudaSuccess) CK(cudaEventRecord(ev, c->stream));
  } else {
    e = coarse_pk_launch(a, cc->g.M, cc->g.N1, c->pk_grid, c->stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    c->pk_failed = true;
    c->pk_grid = 0;
    return false;
  }
  if (trace) {
    std::vector<unsigned long long> ts(nts);
    CK(cudaMemcpyAsync(ts.data(), c->pk_trace, sizeof(unsigned long long) * nts, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    // phases: P0, then per step XF Y Z YI XI (XY Z YXI in the plane form),
    // then the last update, then the sum
    const char *names5[5] = {"XF", "Y", "Z", "YI", "XI"}, *names3[3] = {"XY", "Z", "YXI"};
    const char *const *names = P == 3 ? names3 : names5;
    double ph[7] = {0, 0, 0, 0, 0, 0, 0};
    ph[0] = (double)(ts[1] - ts[0]);
    for (int j = 0; j < k; ++j)
      for (int p = 0; p < P; ++p) ph[1 + p] += (double)(ts[2 + P * j + p] - ts[1 + P * j + p]);
    ph[6] = (double)(ts[P * k + 3] - ts[P * k + 1]);
    std::fprintf(stderr, "pk trace (us): total %.1f  P0 %.1f ", (ts[P * k + 3] - ts[0]) * 1e-3, ph[0] * 1e-3);
    for (int p = 0; p < P; ++p) std::fprintf(stderr, " %s %.1f", names[p], ph[1 + p] * 1e-3);
    std::fprintf(stderr, "  last+sum %.1f (grid %d)\n", ph[6] * 1e-3, c->pk_grid);
    if (trace_ctas) {
      // per phase type: CTA work time (arrival - own previous release),
      // median and max over CTAs and steps; arrival spread (last - first
      // arrival); release lag (last release - last arrival)
      const int G = c->pk_grid;
      std::vector<unsigned long long> tc((size_t)nbar * 2 * G);
      CK(cudaMemcpy(tc.data(), c->pk_trace_cta, sizeof(unsigned long long) * tc.size(), cudaMemcpyDeviceToHost));
      for (int p = 0; p < P; ++p) {
        std::vector<double> work;
        double spread = 0, lag = 0, lagmax = 0;
        for (int j = 0; j < k; ++j) {
          const int b = 1 + P * j + p;  // barrier index (0-based) closing this phase
          unsigned long long amin = ~0ull, amax = 0, rmax = 0;
          for (int q = 0; q < G; ++q) {
            const unsigned long long arr = tc[(size_t)b * 2 * G + q], prev = tc[(size_t)(b - 1) * 2 * G + G + q];
            work.push_back((double)(arr - prev));
            amin = std::min(amin, arr);
            amax = std::max(amax, arr);
            rmax = std::max(rmax, tc[(size_t)b * 2 * G + G + q]);
          }
          spread += (double)(amax - amin);
          lag += (double)(rmax - amax);
          lagmax = std::max(lagmax, (double)(rmax - amax));
        }
        std::sort(work.begin(), work.end());
        std::fprintf(stderr, "  %-2s work median %.2f p90 %.2f max %.2f | arrival spread %.2f | release lag %.2f (max %.2f) us\n",
                     names[p], work[work.size() / 2] * 1e-3, work[work.size() * 9 / 10] * 1e-3, work.back() * 1e-3,
                     spread / k * 1e-3, lag / k * 1e-3, lagmax * 1e-3);
      }
    }
    if (trace_steps) {
      for (int j = 0; j < k; ++j) {
        std::fprintf(stderr, "  step %2d:", j);
        for (int p = 0; p < P; ++p) std::fprintf(stderr, " %6.2f", (ts[2 + P * j + p] - ts[1 + P * j + p]) * 1e-3);
        std::fprintf(stderr, "\n");
      }
    }
  }
  return true;
}

// z = M^-1 (s v).
template <typename T> void tg_apply(rism3d_ctx *c, const T *v, double s, T *z) {
  rism3d_ctx *cc = c->coarse;
  const int prec = sizeof(T) == 8 ? 0 : 1;
  const int k = coarse_steps(c);
  const long long l0 = launch_total(cc);
  {
    TimeScope ts(c, TK_PREC, prec, 6);
    bool done = false;
    if (coarse_pk_ready(c, k)) {
      tg_restrict<T>(c, v, s, basis<float>(cc)[0]);
      done = coarse_pk_run(c, k);
      if (done) {
        c->timer.launches[TK_PREC + 6 * prec] += 1;
        c->coarse_jv += k;
      }
    }
    const bool graph = !done && coarse_graph(c, k);
    c->coarse_driver = done ? 2 : (graph ? 1 : 0);
    if (done) {
    } else if (graph) {
      tg_restrict<T>(c, v, s, basis<float>(cc)[0]);
      CK(cudaGraphLaunch(c->cg_exec, c->stream));
      c->timer.launches[TK_PREC + 6 * prec] += c->cg_nodes;
      c->coarse_jv += k;
    } else {
      tg_restrict<T>(c, v, s, c->tc_r);
      const int jv0 = cc->jv32_evals;
      gmres<float>(cc, slopebuf<float>(cc), c->tc_r, c->tc_y, 0.0, k, k);
      c->coarse_jv += cc->jv32_evals - jv0;
      axpby<float, float>(cc, 1.0, c->tc_r, 1.0, c->tc_y);
    }
    tg_prolong<T>(c, c->tc_y, v, s, z);
  }
  c->timer.launches[TK_PREC + 6 * prec] += launch_total(cc) - l0;
}

template <typename T> std::vector<T *> &zbasis(rism3d_ctx *c);
template <> std::vector<double *> &zbasis<double>(rism3d_ctx *c) { return c->zbasis64; }
template <> std::vector<float *> &zbasis<float>(rism3d_ctx *c) { return c->zbasis32; }

// Flexible GMRES(restart) for J x = b from x0 = 0, right-preconditioned by
// the two-grid M (z_j = M^-1 v_j, x = sum y_j z_j; Saad, SIAM J. Sci.
// Comput. 14 (1993) 461).  Classical Gram-Schmidt as in gmres(); returns
// the number of fine J.v products.
template <typename T>
int fgmres(rism3d_ctx *c, const T *d, const T *b, T *x, double rtol, int maxit, int restart) {
  auto &B = basis<T>(c);
  auto &Z = zbasis<T>(c);
  ensure_basis<T>(c, 1);
  std::vector<double> H((size_t)(restart + 1) * restart), cs(restart), sn(restart), gv(restart + 1);
  std::vector<VecRef<T>> V;
  std::vector<double> h;
  bool have_x = false;
  double beta0 = -1.0;
  int its = 0;
  while (its < maxit) {
    // r0 = b in the first cycle (read in place: the norm-only sweep writes
    // nothing), else B0 = b - J x
    T *r0 = const_cast<T *>(b);
    if (have_x) {
      eval_J<T>(c, d, x, 1.0, B[0], nullptr);  // B0 = J x
      its++;
      xpay<T, T, T>(c, b, -1.0, B[0], B[0]);   // B0 = b - J x
      r0 = B[0];
    }
    const double beta = maxpy<T>(c, r0, 1.0, {}, {}, true);
    if (beta0 < 0) beta0 = beta;
    if (beta == 0.0 || beta <= rtol * beta0) break;
    V.assign(1, vref<T>(r0, 1.0 / beta));
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    int j = 0;
    bool done = false;
    for (; j < restart && its < maxit; ++j) {
      ensure_basis<T>(c, j + 2);
      while ((int)Z.size() <= j) Z.push_back(dalloc<T>(c->nvec));
      tg_apply<T>(c, V[j].p, V[j].s, Z[j]);
      eval_J<T>(c, d, Z[j], 1.0, B[j + 1], nullptr);
      its++;
      double hn;
      if ((int)V.size() <= kVecMax) {
        hn = gs_step<T>(c, B[j + 1], V, h);
      } else {
        mdot<T>(c, B[j + 1], 1.0, V, h);
        hn = maxpy<T>(c, B[j + 1], 1.0, V, h, true);
      }
      for (int i = 0; i <= j; ++i) H[(size_t)i * restart + j] = h[i];
      H[(size_t)(j + 1) * restart + j] = hn;
      for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * restart + j], bb = H[(size_t)(i + 1) * restart + j];
        H[(size_t)i * restart + j] = cs[i] * a + sn[i] * bb;
        H[(size_t)(i + 1) * restart + j] = -sn[i] * a + cs[i] * bb;
      }
      const double a = H[(size_t)j * restart + j], bb = H[(size_t)(j + 1) * restart + j];
      const double r = std::hypot(a, bb);
      cs[j] = r == 0.0 ? 1.0 : a / r;
      sn[j] = r == 0.0 ? 0.0 : bb / r;
      H[(size_t)j * restart + j] = r;
      H[(size_t)(j + 1) * restart + j] = 0.0;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      V.push_back(vref<T>(B[j + 1], hn > 0.0 ? 1.0 / hn : 0.0));
      if (std::fabs(gv[j + 1]) <= rtol * beta0 || hn == 0.0) { ++j; done = true; break; }
    }
    const int k = j;
    std::vector<double> y(k);
    for (int i = k - 1; i >= 0; --i) {
      double s = gv[i];
      for (int l = i + 1; l < k; ++l) s -= H[(size_t)i * restart + l] * y[l];
      y[i] = H[(size_t)i * restart + i] != 0.0 ? s / H[(size_t)i * restart + i] : 0.0;
    }
    std::vector<VecRef<T>> Zk;
    std::vector<double> my(k);
    for (int i = 0; i < k; ++i) {
      Zk.push_back(vref<T>(Z[i], 1.0));
      my[i] = -y[i];
    }
    maxpy<T>(c, x, have_x ? 1.0 : 0.0, Zk, my, false);
    have_x = true;
    if (done) break;
  }
  if (!have_x) axpby<T, T>(c, 0.0, b, 0.0, x);
  return its;
}

struct NewtonOut {
  int iters = 0;
  double rinf = 0, r2 = 0;
  bool converged = false;
  bool nan = false;
  bool stalled = false;
};

// Inexact Newton with backtracking (SNESNEWTONLS, bgy3d-snes.c:160-346):
// state and residual in TS, Jacobian products and Krylov basis in TJ.
// Stops when ||F||_inf < tol.
template <typename TS, typename TJ>
NewtonOut newton(rism3d_ctx *c, TS *x, double tol, int max_iter, double krylov_rtol, int restart,
                 double eta0 = 0.5) {
  NewtonOut o;
  // An accepted step swaps the state with the trial and the residual with
  // the trial residual (pointers, not copies); the state ends in x.
  TS *xc = x;
  TS *F = xbuf<TS>(c, 0);
  TS *xt = xbuf<TS>(c, 1);
  TS *Ft = xbuf<TS>(c, 2);
  TJ *d = slopebuf<TJ>(c);
  TJ *dx = dxbuf<TJ>(c);
  // -F in the Jacobian precision where that differs from the state's (the
  // idle FP32 trial buffer); otherwise the Krylov solve reads F itself and
  // the step is taken with the opposite sign: a solve from zero is odd in
  // its right-hand side, bitwise (negation is exact, every operation
  // sign-symmetric), so dx(F) = -dx(-F)
  constexpr bool same = sizeof(TJ) == sizeof(TS);
  TJ *rhs = same ? nullptr : xbuf<TJ>(c, 1);
  const double sg = same ? -1.0 : 1.0;
  double r[2];
  eval_F<TS>(c, xc, F, r);
  // Eisenstat-Walker forcing (PETSc's version 2: gamma 0.9, alpha 2,
  // safeguard above 0.1), floored at the reference's fixed KSP rtol and
  // never below what the last step needs to reach tol.
  double eta = eta0, r2_prev = -1.0;
  for (int it = 0;; ++it) {
    o.rinf = r[0];
    o.r2 = r[1];
    if (c->pd.verbosity > 0)
      std::fprintf(stderr, " # newton<%s,%s> %3d: |F|inf = %.3e |F|2 = %.3e\n", sizeof(TS) == 8 ? "f64" : "f32",
                   sizeof(TJ) == 8 ? "f64" : "f32", it, r[0], r[1]);
    if (!(r[0] == r[0]) || !(r[1] == r[1]) || std::isinf(r[0])) { o.nan = true; break; }
    if (r[0] < tol) { o.converged = true; break; }
    if (it >= max_iter) break;
    o.iters = it + 1;
    if (r2_prev > 0.0) {
      const double ratio = r[1] / r2_prev;
      double e = 0.9 * ratio * ratio;
      const double guard = 0.9 * eta * eta;
      if (guard > 0.1) e = std::max(e, guard);
      eta = std::min(0.9, e);
    }
    double eta_use = c->pd.ew_forcing ? std::max(std::max(eta, krylov_rtol), std::min(0.9, 0.5 * tol / r[0]))
                                      : krylov_rtol;
    // With the two-grid preconditioner a loose forcing term is met after one
    // or two iterations by a direction taken mostly from the coarse
    // Jacobian, which far from the root of an HNC problem can be a poor
    // descent direction (the line search then creeps).  Preconditioned
    // iterations are cheap, so those solves are held to 0.1.
    if (c->coarse) eta_use = std::min(eta_use, 0.1);
    r2_prev = r[1];
    closure_slope<TS, TJ>(c, xc, d);
    const TJ *b;
    if constexpr (same) {
      b = F;
    } else {
      axpby<TS, TJ>(c, -1.0, F, 0.0, rhs);
      b = rhs;
    }
    int kits;
    if (c->coarse) {
      tg_prepare<TJ>(c, d);
      kits = fgmres<TJ>(c, d, b, dx, eta_use, 1000, restart);
    } else {
      kits = gmres<TJ>(c, d, b, dx, eta_use, 1000, restart);
    }
    if (c->pd.verbosity > 0) std::fprintf(stderr, "   gmres: %d J.v (rtol %.2e)\n", kits, eta_use);
    const double f0 = r[1] * r[1];
    double lam = 1.0, f1 = 0.0, rt[2] = {0, 0};
    bool decreased = false;
    for (int ls = 0; ls < 20; ++ls) {
      xpay<TS, TJ, TS>(c, xc, sg * lam, dx, xt);
      eval_F<TS>(c, xt, Ft, rt);
      f1 = rt[1] * rt[1];
      if (f1 <= (1.0 - 2e-4 * lam) * f0) { decreased = true; break; }
      if (!(f1 == f1)) break;
      double ln = lam * lam * f0 / (f1 - f0 + 2.0 * lam * f0);
      ln = std::min(std::max(ln, 0.1 * lam), 0.5 * lam);
      lam = ln;
    }
    if (!decreased) {  // SNES_DIVERGED_LINE_SEARCH: keep the last accepted x
      o.stalled = true;
      break;
    }
    // accept: the trial becomes the state, its residual the residual
    std::swap(xc, xt);
    std::swap(F, Ft);
    r[0] = rt[0];
    r[1] = rt[1];
  }
  if (xc != x) axpby<TS, TS>(c, 1.0, xc, 0.0, x);
  return o;
}

int solve_impl(rism3d_ctx *c, double *T, rism3d_result *out) {
  rism3d_result res{};
  c->f_evals = c->jv_evals = c->f32_evals = c->jv32_evals = 0;
  c->coarse_jv = 0;
  const long long launches0 = launch_total(c);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c->stream));
  const double krtol = 1e-3;  // 100 * PETSc default rtol 1e-5 (bgy3d-snes.c:277)
  const int restart = c->pd.krylov_restart > 0 ? std::min(c->pd.krylov_restart, 200) : 30;
  NewtonOut o;
  int status = RISM3D_OK;
  const rism3d_problem &pd = c->pd;
  const bool mixing = pd.solver == RISM3D_PICARD || pd.solver == RISM3D_JAGER;  // no Jacobian
  if (pd.closure == RISM3D_PY && !mixing) {
    CK(cudaEventDestroy(e0));
    CK(cudaEventDestroy(e1));
    return RISM3D_ERR_UNSUPPORTED;
  }
  if (pd.solver == RISM3D_PICARD || pd.solver == RISM3D_TRIAL) {
    // bgy3d_snes_picard (bgy3d-snes.c:348-384): x += lambda F(x).
    const int steps = pd.solver == RISM3D_TRIAL ? 100 : pd.max_iter;
    const double lam = pd.solver == RISM3D_TRIAL ? 0.02 : pd.lambda;
    double *F = xbuf<double>(c, 0);
    double r[2] = {0, 0};
    for (int k = 0; k < steps; ++k) {
      eval_F<double>(c, T, F, r);
      xpay<double, double, double>(c, T, lam, F, T);
      o.iters = k + 1;
      if (r[0] < pd.norm_tol) { o.converged = true; break; }
    }
    o.rinf = r[0];
    o.r2 = r[1];
  }
  if (pd.solver == RISM3D_JAGER) {
    // bgy3d_snes_jager (bgy3d-snes.c:402-509): x += a F(x), where a is the
    // "move" coefficient a1 every 10th iteration and lambda otherwise; a1
    // doubles (up to 1) after 20 quiet iterations and halves (down to
    // lambda) when a move made an otherwise falling norm go up.
    const double a0 = pd.lambda;
    double a1 = pd.lambda, norm_old = 0.0;
    int mycount = 0, upwards = 0;
    const int nth = 10;
    double *F = xbuf<double>(c, 0);
    double r[2] = {0, 0};
    for (int iter = 0; iter < pd.max_iter; ++iter) {
      eval_F<double>(c, T, F, r);
      const double norm = r[0];
      const double a = (iter % nth == 0) ? a1 : a0;
      xpay<double, double, double>(c, T, a, F, T);
      const bool up = norm > norm_old;
      norm_old = norm;
      mycount++;
      if (iter % nth != 1) upwards = up ? 1 : 0;
      if (iter % nth == 1 && up && upwards == 0 && iter > 2 * nth) {
        a1 = std::max(a1 / 2.0, a0);
        mycount = 0;
      }
      if (mycount > 2 * nth) {
        a1 = std::min(a1 * 2.0, 1.0);
        mycount = 0;
      }
      o.iters = iter + 1;
      if (!(norm == norm)) { o.nan = true; break; }
      if (norm <= pd.norm_tol) { o.converged = true; break; }
    }
    o.rinf = r[0];
    o.r2 = r[1];
  }
  if (!mixing) {
    if (pd.precision == RISM3D_MIXED) {
      // FP32 bulk: Newton on a float copy of t until the float residual floor.
      if (!c->X32) c->X32 = dalloc<float>(c->nvec);
      axpby<double, float>(c, 1.0, T, 0.0, c->X32);
      const double tol32 = std::max(pd.norm_tol, 2e-4);
      NewtonOut a = newton<float, float>(c, c->X32, tol32, pd.max_iter, krtol, restart);
      axpby<float, double>(c, 1.0, c->X32, 0.0, T);
      // FP64 residual with FP32 Jacobian: iterative refinement to norm_tol.
      o = newton<double, float>(c, T, pd.norm_tol, pd.max_iter, krtol, restart, krtol);
      o.iters += a.iters;
    } else {
      o = newton<double, double>(c, T, pd.norm_tol, pd.max_iter, krtol, restart);
    }
  }
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  CK(cudaEventDestroy(e0));
  CK(cudaEventDestroy(e1));
  if (o.nan) status = RISM3D_ERR_NAN;
  else if (!o.converged) status = RISM3D_ERR_NOT_CONVERGED;
  res.status = status;
  res.newton_iters = o.iters;
  res.resid_inf = o.rinf;
  res.resid_2 = o.r2;
  res.f_evals = c->f_evals;
  res.jv_evals = c->jv_evals;
  res.f_evals_fp32 = c->f32_evals;
  res.jv_evals_fp32 = c->jv32_evals;
  res.jv_evals_coarse = c->coarse_jv;
  res.launches = launch_total(c) - launches0;
  res.seconds = ms * 1e-3;
  if (out) {
    const double keep[5] = {out->mu, out->mu_hnc, out->mu_kh, out->mu_gf, out->pmv_factor};
    *out = res;
    out->mu = keep[0]; out->mu_hnc = keep[1]; out->mu_kh = keep[2]; out->mu_gf = keep[3];
    out->pmv_factor = keep[4];
  }
  return status;
}

int observables_impl(rism3d_ctx *c, const double *T, double *g, rism3d_result *out) {
  const Geo &G = c->g;
  const rism3d_problem &pd = c->pd;
  const double h0 = pd.L[0] / pd.N[0], h1 = pd.L[1] / pd.N[1], h2 = pd.L[2] / pd.N[2];
  const unsigned nb = (unsigned)((G.Nr + 255) / 256);
  // the solute's long-range Coulomb field: computed once per bound solute
  if (!c->uc64) c->uc64 = dalloc<double>(G.Nr);
  if (!c->uc_valid) {
    k_coulomb_long<<<nb, 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], c->n, c->d_solute, c->uc64);
    CKL();
    c->uc_valid = true;
    c->timer.launches[TK_VEC] += 1;
  }
  ObsPartial *part = dalloc<ObsPartial>(nb);
  k_observables<<<nb, 256, 0, c->stream>>>(G, T, c->v64, c->uc64, pd.beta, pd.closure, c->d_charge, g, part);
  CKL();
  // the five sums reduced on the device in a fixed order; five doubles to
  // pinned host memory
  double *dsum = c->dres + 3 * kVecMax;
  k_obs_final<<<1, 1024, 0, c->stream>>>(nb, part, dsum);
  CKL();
  c->timer.launches[TK_VEC] += 2;
  double *s = pinned_scratch();
  CK(cudaMemcpyAsync(s, dsum, sizeof(double) * 5, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  dfree(part);
  // mu = rho * sum * h^3 / beta (chempot, hnc3d.c:604-623); PMV 1 - rho h^3 sum c
  const double f = pd.rho * c->h3 / pd.beta;
  if (out) {
    out->mu = s[0] * f;
    out->mu_hnc = s[1] * f;
    out->mu_kh = s[2] * f;
    out->mu_gf = s[3] * f;
    out->pmv_factor = 1.0 - s[4] * (pd.rho * c->h3);
  }
  return RISM3D_OK;
}

// ------------------------------------------------------------- gradient
// Plain forward 3D transform of an FP64 field into W (runtime-length passes).
void fwd3d(rism3d_ctx *c, const double *A) {
  const Geo &G = c->g;
  auto *W = c->work<double>();
  const TileShape &t = c->tl<double>();
  dim3 gx((G.N1 * G.N2 + t.RX - 1) / t.RX, c->m);
  k_xfwd<double, MODE_FWD><<<gx, 256, xsmem<double>(c), c->stream>>>(G, c->plan<double>(0), t.RX, A, A, 1.0,
                                                                     c->pd.closure, W, postw<double>(c));
  CKL();
  dim3 gy((G.Nh + t.BY - 1) / t.BY, G.N2, c->m);
  const size_t sy = ysmem<double>(c);
  if (t.BY == 16) k_y<double, false, 16><<<gy, 256, sy, c->stream>>>(G, c->plan<double>(1), W);
  else if (t.BY == 8) k_y<double, false, 8><<<gy, 256, sy, c->stream>>>(G, c->plan<double>(1), W);
  else k_y<double, false, 4><<<gy, 256, sy, c->stream>>>(G, c->plan<double>(1), W);
  CKL();
  dim3 gz((G.Nh + t.BZ - 1) / t.BZ, G.N1);
  const size_t sz = zsmem<double>(c);
  const ZParams<double> zp = zparams<double>(c, false);
  if (t.BZ == 16) k_z<double, MODE_FWD, 16><<<gz, 256, sz, c->stream>>>(G, c->plan<double>(2), W, zp);
  else if (t.BZ == 8) k_z<double, MODE_FWD, 8><<<gz, 256, sz, c->stream>>>(G, c->plan<double>(2), W, zp);
  else k_z<double, MODE_FWD, 4><<<gz, 256, sz, c->stream>>>(G, c->plan<double>(2), W, zp);
  CKL();
  c->timer.launches[TK_XFWD] += 3;
}

// out = K v = (chi - 1) * v (the OZ convolution alone): the J.v passes with
// unit slope and nothing subtracted.
void kconv(rism3d_ctx *c, const double *ones, const double *v, double *out) {
  pipeline<double, MODE_J>(c, v, ones, 1.0, 0.0, out);
}

double *ones_field(rism3d_ctx *c) {
  double *o = dalloc<double>(c->nvec);
  k_fill<<<vec_grid(c->nvec), 256, 0, c->stream>>>(c->nvec, 1.0, o);
  CKL();
  return o;
}

int jacobian_transpose_impl(rism3d_ctx *c, const double *T, const double *dT, double *out) {
  double *d = slopebuf<double>(c);
  closure_slope<double, double>(c, T, d);
  double *ones = ones_field(c);
  double *kv = dalloc<double>(c->nvec);
  kconv(c, ones, dT, kv);
  k_dmul_sub<<<vec_grid(c->nvec), 256, 0, c->stream>>>(c->nvec, d, kv, dT, out);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  dfree(kv);
  dfree(ones);
  return RISM3D_OK;
}

// dmu/d(q, sigma, eps, x) of every solute site at the converged T.  The
// adjoint J^T lambda = b (b = dmu/dt) is solved through the forward
// Jacobian: with J = K D - 1 and J^T = D K - 1, lambda = D y - b where
// J y = K b, so the preconditioned FGMRES of the Newton steps serves.
int gradient_impl(rism3d_ctx *c, const double *T, rism3d_grad *gr) {
  const rism3d_problem &pd = c->pd;
  if (!pd.renorm) {
    g_last_error = "the gradient is implemented for the renormalised form only";
    return RISM3D_ERR_UNSUPPORTED;
  }
  const Geo &G = c->g;
  const long long nv = c->nvec;
  const double h0 = pd.L[0] / pd.N[0], h1 = pd.L[1] / pd.N[1], h2 = pd.L[2] / pd.N[2];
  const double rhoh3 = pd.rho * c->h3, rhoh3b = rhoh3 / pd.beta;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c->stream));
  const unsigned nb = (unsigned)((G.Nr + 255) / 256);
  double *uc = dalloc<double>(G.Nr);
  k_coulomb_long<<<nb, 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], c->n, c->d_solute, uc);
  CKL();
  double *d = slopebuf<double>(c);
  closure_slope<double, double>(c, T, d);
  double *ones = ones_field(c);
  double *b = dalloc<double>(nv), *y = dalloc<double>(nv), *w = dalloc<double>(nv), *Bw = dalloc<double>(G.Nr);
  k_mu_dt<<<nb, 256, 0, c->stream>>>(G, T, c->v64, uc, pd.beta, pd.closure, c->d_charge, rhoh3b, b);
  CKL();
  const double bnorm = maxpy<double>(c, b, 1.0, {}, {}, true);
  // J y = K b; lambda = d y - b (into w)
  kconv(c, ones, b, w);
  const int restart = pd.krylov_restart > 0 ? std::min(pd.krylov_restart, 200) : 30;
  const int jv0 = c->jv_evals;
  if (c->coarse) {
    tg_prepare<double>(c, d);
    fgmres<double>(c, d, w, y, 1e-11, 4000, restart);
  } else {
    gmres<double>(c, d, w, y, 1e-11, 4000, restart);
  }
  gr->adjoint_jv = c->jv_evals - jv0;
  k_dmul_sub<<<vec_grid(nv), 256, 0, c->stream>>>(nv, d, y, b, w);
  CKL();
  double *lam = w;
  // K lambda (into y); adjoint residual d K lambda - lambda - b (into b)
  kconv(c, ones, lam, y);
  k_dmul_sub<<<vec_grid(nv), 256, 0, c->stream>>>(nv, d, y, lam, ones);  // ones <- J^T lambda
  CKL();
  xpay<double, double, double>(c, ones, -1.0, b, b);  // b <- J^T lambda - b
  gr->adjoint_resid = bnorm > 0 ? maxpy<double>(c, b, 1.0, {}, {}, true) / bnorm : 0.0;
  // weights A (into b, m fields) and B; real-space sums
  k_grad_weights<<<nb, 256, 0, c->stream>>>(G, T, c->v64, uc, y, pd.beta, pd.closure, c->d_charge, rhoh3b, rhoh3,
                                            b, Bw);
  CKL();
  const int n = c->n;
  std::vector<double> gq(n, 0.0), gs(n, 0.0), ge(n, 0.0), gx(3 * (size_t)n, 0.0);
  if (n > 0) {
    const int rb = (int)std::min<long long>(2 * 148, (G.Nr + 255) / 256);
    double *part = dalloc<double>((size_t)rb * n * 6);
    k_grad_real<<<dim3(rb, n), 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], c->d_solvent,
                                                    c->d_solute, b, Bw, part);
    CKL();
    std::vector<double> hp((size_t)rb * n * 6);
    CK(cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, c->stream));
    // tau term: FFT lambda, then the half-spectrum sums
    fwd3d(c, lam);
    const long long nk = (long long)G.Nh * G.N1 * G.N2;
    const int kb = (int)std::min<long long>(2 * 148, (nk + 255) / 256);
    double *kpart = dalloc<double>((size_t)kb * n * 4);
    k_grad_kspace<<<dim3(kb, n), 256, 0, c->stream>>>(G, c->work<double>(), c->s64, pd.nrad, c->dkr, c->d_solute,
                                                      kpart);
    CKL();
    std::vector<double> hk((size_t)kb * n * 4);
    CK(cudaMemcpyAsync(hk.data(), kpart, sizeof(double) * hk.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    dfree(part);
    dfree(kpart);
    const double kf = 1.0 / ((double)G.Nr * c->h3);
    for (int u = 0; u < n; ++u) {
      double a[6] = {0, 0, 0, 0, 0, 0}, k4[4] = {0, 0, 0, 0};
      for (int q = 0; q < rb; ++q)
        for (int j = 0; j < 6; ++j) a[j] += hp[((size_t)u * rb + q) * 6 + j];
      for (int q = 0; q < kb; ++q)
        for (int j = 0; j < 4; ++j) k4[j] += hk[((size_t)u * kb + q) * 4 + j];
      gq[u] = a[0] + kf * k4[0];
      gs[u] = a[1];
      ge[u] = a[2];
      for (int j = 0; j < 3; ++j) gx[3 * (size_t)u + j] = a[3 + j] + kf * k4[1 + j];
    }
  }
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  gr->seconds = ms * 1e-3;
  for (double *p : {b, y, w, Bw, uc, ones}) dfree(p);
  if (gr->dq) std::copy(gq.begin(), gq.end(), gr->dq);
  if (gr->dsigma) std::copy(gs.begin(), gs.end(), gr->dsigma);
  if (gr->depsilon) std::copy(ge.begin(), ge.end(), gr->depsilon);
  if (gr->dx) std::copy(gx.begin(), gx.end(), gr->dx);
  return RISM3D_OK;
}

// Linear-response dmu/dR (the response branch of hnc3d_solute_solve): one
// preconditioned FGMRES solve J dT = beta K((c' + 1) dv) per unit
// displacement, then the free-energy differential reduced on the device.
int response_impl(rism3d_ctx *c, const double *T, rism3d_grad *gr) {
  const rism3d_problem &pd = c->pd;
  if (pd.closure == 2) {
    g_last_error = "PY has no closure differential";
    return RISM3D_ERR_UNSUPPORTED;
  }
  const Geo &G = c->g;
  const long long nv = c->nvec;
  const double h0 = pd.L[0] / pd.N[0], h1 = pd.L[1] / pd.N[1], h2 = pd.L[2] / pd.N[2];
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c->stream));
  const unsigned nb = (unsigned)((G.Nr + 255) / 256);
  double *uc = dalloc<double>(G.Nr);
  k_coulomb_long<<<nb, 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], c->n, c->d_solute, uc);
  CKL();
  double *d = slopebuf<double>(c);
  closure_slope<double, double>(c, T, d);
  double *d1 = dalloc<double>(nv), *dv = dalloc<double>(nv), *B = dalloc<double>(nv), *dT = dalloc<double>(nv);
  double *Bc = dalloc<double>(nv);
  k_shift1<<<vec_grid(nv), 256, 0, c->stream>>>(nv, d, d1);
  CKL();
  const int restart = pd.krylov_restart > 0 ? std::min(pd.krylov_restart, 200) : 30;
  if (c->coarse) tg_prepare<double>(c, d);
  const int n = c->n;
  const int rb = (int)std::min<long long>(2 * 148, (G.Nr + 255) / 256);
  double *part = dalloc<double>((size_t)rb * 3 * std::max(n, 1));
  const int jv0 = c->jv_evals;
  double worst = 0.0;
  for (int u = 0; u < n; ++u)
    for (int dim = 0; dim < 3; ++dim) {
      k_field1<<<nb, 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], c->d_solvent, c->d_solute, u,
                                          dim, dv);
      CKL();
      // B = beta (chi - 1) * ((c' + 1) dv): the Jacobian passes with slope
      // c' + 1 and nothing subtracted (jacobian_t1 with its flag set)
      pipeline<double, MODE_J>(c, dv, d1, pd.beta, 0.0, B);
      const double bnorm = maxpy<double>(c, B, 1.0, {}, {}, true);
      axpby<double, double>(c, 1.0, B, 0.0, Bc);  // the solvers may overwrite B
      if (c->coarse) fgmres<double>(c, d, B, dT, 1e-11, 4000, restart);
      else gmres<double>(c, d, B, dT, 1e-11, 4000, restart);
      k_mu1<<<rb, 256, 0, c->stream>>>(G, T, c->v64, uc, dv, dT, pd.beta, pd.closure, c->d_charge,
                                       part + (size_t)(3 * u + dim) * rb);
      CKL();
      // true residual of the solve: B - J dT (into dv, no longer needed)
      eval_J<double>(c, d, dT, 1.0, dv, nullptr);
      xpay<double, double, double>(c, Bc, -1.0, dv, dv);
      const double rn = maxpy<double>(c, dv, 1.0, {}, {}, true);
      if (bnorm > 0) worst = std::max(worst, rn / bnorm);
    }
  gr->adjoint_jv = c->jv_evals - jv0;
  gr->adjoint_resid = worst;
  std::vector<double> hp((size_t)rb * 3 * n);
  if (n > 0)
    CK(cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  gr->seconds = ms * 1e-3;
  for (double *p : {d1, dv, B, Bc, dT, uc, part}) dfree(p);
  // mu1 = rho h^3 / beta * sum (chempot1, hnc3d.c:627-650)
  const double f = pd.rho * c->h3 / pd.beta;
  if (gr->dx)
    for (int q = 0; q < 3 * n; ++q) {
      double a = 0.0;
      for (int b = 0; b < rb; ++b) a += hp[(size_t)q * rb + b];
      gr->dx[q] = a * f;
    }
  return RISM3D_OK;
}

// The reference's free-energy gradient at T (the `derivatives` output,
// hnc3d.c:1665-1742): de[n][3] = rho h^3 sum_i <g_i, dv_i/dR_u> with the
// field1 derivative, reduced on the device; any context (renormalised or
// not, radial or 3D chi).  Host de, may be NULL (the sums are still made).
int reference_gradient_impl(rism3d_ctx *c, const double *T, double *de) {
  const rism3d_problem &pd = c->pd;
  const Geo &G = c->g;
  const int n = c->n;
  if (c->pure) {
    g_last_error = "the free-energy gradient needs a solute context";
    return RISM3D_ERR_UNSUPPORTED;
  }
  if (n == 0) return RISM3D_OK;
  constexpr int U = 4;
  const double h0 = pd.L[0] / pd.N[0], h1 = pd.L[1] / pd.N[1], h2 = pd.L[2] / pd.N[2];
  const int rb = (int)std::min<long long>(2 * 148, (G.Nr + 255) / 256);
  double *part = dalloc<double>((size_t)rb * n * 3);
  struct Free { double *p; ~Free() { dfree(p); } } fr{part};
  k_force_pair<U><<<dim3(rb, (n + U - 1) / U), 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2],
                                                                     c->d_solvent, n, c->d_solute, T, c->v64,
                                                                     pd.beta, pd.closure, part);
  CKL();
  std::vector<double> hp((size_t)rb * n * 3);
  CK(cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const double dN = pd.rho * c->h3;
  for (int u = 0; u < n; ++u)
    for (int d = 0; d < 3; ++d) {
      double a = 0.0;
      for (int q = 0; q < rb; ++q) a += hp[((size_t)u * rb + q) * 3 + d];
      if (de) de[3 * u + d] = dN * a;
    }
  return RISM3D_OK;
}

// (Re)binds the solute: its device copy, the short-range field v (FP64 and
// FP32) and the long-range field L; grid, chi tables and work buffers stay.
void bind_solute(rism3d_ctx *c, int n, const rism3d_site *solute) {
  const Geo &G = c->g;
  const rism3d_problem &pd = c->pd;
  c->uc_valid = false;  // the observables' Coulomb field follows the solute
  std::vector<SiteP> hs(std::max(n, 1));
  for (int u = 0; u < n; ++u)
    hs[u] = SiteP{solute[u].x[0], solute[u].x[1], solute[u].x[2], solute[u].sigma, solute[u].epsilon,
                  solute[u].charge};
  if (!c->d_solute || n > c->n_cap) {
    dfree(c->d_solute);
    c->n_cap = std::max(n, 1);
    c->d_solute = dalloc<SiteP>(c->n_cap);
  }
  CK(cudaMemcpyAsync(c->d_solute, hs.data(), sizeof(SiteP) * std::max(n, 1), cudaMemcpyHostToDevice, c->stream));
  c->n = n;
  c->solute.assign(solute, solute + n);
  const double h0 = pd.L[0] / pd.N[0], h1 = pd.L[1] / pd.N[1], h2 = pd.L[2] / pd.N[2];
  const unsigned nb = (unsigned)((G.Nr + 255) / 256);
  if (n * G.m <= kField0MaxPairs && n <= 384) {
    const size_t sm = sizeof(double) * (size_t)(4 * n * G.m + 3 * n);
    k_field0_pairs<<<nb, 256, sm, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], c->d_solvent, n,
                                               c->d_solute, c->v64);
  } else {
    k_field0<<<nb, 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], c->d_solvent, n, c->d_solute,
                                        c->v64);
  }
  CKL();
  k_axpby<double, float><<<vec_grid(c->nvec), 256, 0, c->stream>>>(c->nvec, 1.0, c->v64, 0.0, c->v32);
  CKL();
  CK(cudaMemsetAsync(c->L64, 0, sizeof(double2) * (size_t)G.Nhp * G.N1 * G.N2, c->stream));
  CK(cudaMemsetAsync(c->L32, 0, sizeof(float2) * (size_t)G.Nhp * G.N1 * G.N2, c->stream));
  const long long nk = (long long)G.Nh * G.N1 * G.N2;
  // per-axis phase tables of the solute form factor, then the k-field
  const size_t per = (size_t)G.Nh + G.N1 + G.N2;
  if (!c->phase_tab || n > c->phase_cap) {
    dfree(c->phase_tab);
    c->phase_cap = std::max(n, 1);
    c->phase_tab = dalloc<double2>((size_t)c->phase_cap * per);
  }
  double2 *t0 = c->phase_tab, *t1 = t0 + (size_t)c->phase_cap * G.Nh, *t2 = t1 + (size_t)c->phase_cap * G.N1;
  if (n > 0) {
    k_phase_axis<<<(n * G.Nh + 255) / 256, 256, 0, c->stream>>>(n, G.Nh, G.N0, G.dk0, 0, c->d_solute, t0);
    k_phase_axis<<<(n * G.N1 + 255) / 256, 256, 0, c->stream>>>(n, G.N1, G.N1, G.dk1, 1, c->d_solute, t1);
    k_phase_axis<<<(n * G.N2 + 255) / 256, 256, 0, c->stream>>>(n, G.N2, G.N2, G.dk2, 2, c->d_solute, t2);
    CKL();
  }
  k_longrange_tab<<<(unsigned)((nk + 255) / 256), 256, 0, c->stream>>>(G, n, c->d_solute, t0, t1, t2, pd.renorm,
                                                                       1.0 / c->h3, c->L64, c->L32);
  CKL();
  CK(cudaStreamSynchronize(c->stream));  // hs is freed on return
  if (c->coarse) bind_solute(c->coarse, n, solute);
}

// ------------------------------------------------------------ autotuner
// The batch sizes of the runtime-length passes (x rows, y and z columns per
// CTA) and, where shape-specialised passes exist, the choice between them and
// the runtime-length ones are timed on the context's own buffers the first
// time a (grid, fields) shape is seen in the process; the winners are cached.
// Only the scheduling changes: every candidate computes the same transforms
// column by column.  RISM3D_AUTOTUNE=0 keeps the register / occupancy rule.
struct TuneVal {
  TileShape t[2];
  bool stat[2];
  int zb[2];
  bool zpers[2];
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, TuneVal> g_tune;

int optin_limit() {
  int dev = 0, optin = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  return optin - 4096;  // margin for the kernels' static shared memory
}

template <typename F> float time_ms(rism3d_ctx *c, F &&f, int reps) {
  f();  // warm
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, c->stream));
  for (int i = 0; i < reps; ++i) f();
  CK(cudaEventRecord(b, c->stream));
  CK(cudaEventSynchronize(b));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

template <typename T> void tune_precision(rism3d_ctx *c, const T *A, const T *Bv, T *out) {
  const int pr = sizeof(T) == 8 ? 0 : 1;
  const Geo &G = c->g;
  TileShape &t = c->tiles[pr];
  const int rc = pr == 0 ? reg_complex<double2>() : reg_complex<float2>();
  const size_t cs = sizeof(typename Cx<T>::type);
  const long long lim = optin_limit();
  const int reps = G.Nr >= (1LL << 22) ? 2 : 5;
  const bool had_stat = c->stat[pr];
  c->stat[pr] = false;
  auto run = [&] { pipeline<T, MODE_J>(c, A, Bv, (T)1, (T)1, out); };
  const int cand[4] = {4, 8, 16, 32};
  // one axis at a time, the others held
  int *fields[3] = {&t.RX, &t.BY, &t.BZ};
  for (int axis = 0; axis < 3; ++axis) {
    int best = *fields[axis];
    float best_ms = time_ms(c, run, reps);
    for (int k : cand) {
      if (k == best) continue;
      long long smem;
      if (axis == 0) {
        if (G.M * k > rc * 256 || (k > 16)) continue;
        smem = (long long)cs * (G.M + k * G.M);
      } else if (axis == 1) {
        if (G.N1 * k > rc * 256 || k > 16) continue;
        smem = (long long)cs * (G.N1 + G.N1 * k);
      } else {
        if (G.N2 * k > rc * 256 || k > 16) continue;
        smem = (long long)cs * (G.N2 + (long long)G.N2 * G.m * k);
      }
      if (smem > lim) continue;
      const int keep = *fields[axis];
      *fields[axis] = k;
      const float ms = time_ms(c, run, reps);
      if (ms < 0.97f * best_ms) { best_ms = ms; best = k; }  // a clear win only: timings are noisy
      *fields[axis] = keep;
    }
    *fields[axis] = best;
  }
  if (had_stat) {
    const float g_ms = time_ms(c, run, reps);
    c->stat[pr] = true;
    float s_ms = time_ms(c, run, reps);
    // the specialised z pass: wide tiles, or half as wide (twice the CTAs
    // in flight per SM)
    const int wide = c->zb[pr];
    float n_ms = 1e30f;
    if (pr == 1) {  // FP32 only: 64-byte rows (FP64 would drop to 32-thread CTAs)
      c->zb[pr] = wide / 2;
      make_tmap(c, &c->tmz[pr], pr == 0, c->zb[pr], 1, G.N2);
      n_ms = time_ms(c, run, reps);
    }
    if (n_ms < 0.95f * s_ms) {
      s_ms = n_ms;
    } else {
      c->zb[pr] = wide;
      make_tmap(c, &c->tmz[pr], pr == 0, wide, 1, G.N2);
      // persistent double-buffered CTAs for the wide tiles
      c->zpers[pr] = true;
      const float p_ms = time_ms(c, run, reps);
      if (p_ms < 0.97f * s_ms) s_ms = p_ms;
      else c->zpers[pr] = false;
    }
    c->stat[pr] = s_ms <= 1.05f * g_ms;  // keep the specialised passes unless clearly slower
  }
}

// RISM3D_Z_PERSISTENT=1 / 0 forces the persistent z pass on / off where the
// shape-specialised passes run (the tests compare both).
void force_z_persistent(rism3d_ctx *c) {
  const char *env = std::getenv("RISM3D_Z_PERSISTENT");
  if (!env || (env[0] != '0' && env[0] != '1')) return;
  const int wide[2] = {static_Bz<double>(), static_Bz<float>()};
  for (int pr = 0; pr < 2; ++pr) {
    if (!c->stat[pr]) continue;
    if (c->zb[pr] != wide[pr]) {
      c->zb[pr] = wide[pr];
      make_tmap(c, &c->tmz[pr], pr == 0, wide[pr], 1, c->g.N2);
    }
    c->zpers[pr] = env[0] == '1';
  }
}

// Applies the cached shapes of this context's (grid, fields) or times them.
void autotune(rism3d_ctx *c) {
  struct Force { rism3d_ctx *c; ~Force() { force_z_persistent(c); } } force{c};
  const char *env = std::getenv("RISM3D_AUTOTUNE");
  if (env && env[0] == '0') return;
  const Geo &G = c->g;
  const int kind = c->pure ? 2 : (c->chi3_64 ? 1 : 0);  // the z pass differs per kind
  const auto key = std::make_tuple(G.N0, G.N1, G.N2, G.m, kind);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      for (int pr = 0; pr < 2; ++pr) {
        c->tiles[pr] = it->second.t[pr];
        c->stat[pr] = c->stat[pr] && it->second.stat[pr];
        c->zpers[pr] = c->stat[pr] && it->second.zpers[pr];
        if (c->stat[pr] && c->zb[pr] != it->second.zb[pr]) {
          c->zb[pr] = it->second.zb[pr];
          make_tmap(c, &c->tmz[pr], pr == 0, c->zb[pr], 1, G.N2);
        }
      }
      return;
    }
  }
  const long long nv = c->nvec;
  double *a64 = dalloc<double>(nv), *b64 = dalloc<double>(nv), *o64 = dalloc<double>(nv);
  CK(cudaMemsetAsync(a64, 0, sizeof(double) * nv, c->stream));
  CK(cudaMemsetAsync(b64, 0, sizeof(double) * nv, c->stream));
  tune_precision<double>(c, a64, b64, o64);
  if (!c->pure) {
    float *a32 = reinterpret_cast<float *>(a64), *b32 = reinterpret_cast<float *>(b64);
    tune_precision<float>(c, a32, b32, reinterpret_cast<float *>(o64));
  }
  CK(cudaStreamSynchronize(c->stream));
  dfree(a64);
  dfree(b64);
  dfree(o64);
  c->timer = PassTimer{};
  std::lock_guard<std::mutex> lk(g_tune_mu);
  TuneVal v;
  for (int pr = 0; pr < 2; ++pr) {
    v.t[pr] = c->tiles[pr];
    v.stat[pr] = c->stat[pr];
    v.zb[pr] = c->zb[pr];
    v.zpers[pr] = c->zpers[pr];
  }
  g_tune[key] = v;
}

void check_grid(const rism3d_problem *pd) {
  for (int d = 0; d < 3; ++d) {
    if (!is_2a3b(pd->N[d]) || pd->N[d] % 2 || pd->N[d] < 8 || pd->N[d] > kMaxN)
      throw ArgFail{RISM3D_ERR_ARG, "N must be even 2^a 3^b in [8, 512]"};
    if (!(pd->L[d] > 0)) throw ArgFail{RISM3D_ERR_ARG, "L must be positive"};
  }
  if (pd->closure < 0 || pd->closure > RISM3D_PSE7) throw ArgFail{RISM3D_ERR_ARG, "no such closure"};
}

// Geometry, tile shapes, FFT plans and twiddles of a context over `fields`
// real fields on the grid of c->pd.
void init_grid(rism3d_ctx *c, int fields) {
  const rism3d_problem *pd = &c->pd;
  Geo &G = c->g;
  G.N0 = pd->N[0]; G.N1 = pd->N[1]; G.N2 = pd->N[2];
  G.M = G.N0 / 2;
  G.Nh = G.M + 1;
  G.Nhp = (G.Nh + 1) & ~1;
  G.m = fields;
  G.Nr = (long long)G.N0 * G.N1 * G.N2;
  G.Nc = (long long)G.Nhp * G.N1 * G.N2;
  const double pi = 3.14159265358979323846;
  G.dk0 = 2 * pi / pd->L[0];
  G.dk1 = 2 * pi / pd->L[1];
  G.dk2 = 2 * pi / pd->L[2];
  c->nvec = (long long)fields * G.Nr;
  const double h0 = pd->L[0] / pd->N[0], h1 = pd->L[1] / pd->N[1], h2 = pd->L[2] / pd->N[2];
  c->h3 = h0 * h1 * h2;
  c->dkr = pd->rmax > 0 ? pi / pd->rmax : 0.0;
  const int m = fields;
  // tile shapes per precision: n * batch <= reg_complex * 256 threads
  for (int pr = 0; pr < 2; ++pr) {
    const int rc = pr == 0 ? reg_complex<double2>() : reg_complex<float2>();
    TileShape &t = c->tiles[pr];
    t.RX = 32;
    while (t.RX > 1 && G.M * t.RX > rc * 256) t.RX /= 2;
    t.BY = 16;
    while (t.BY > 4 && G.N1 * t.BY > rc * 256) t.BY /= 2;
    t.BZ = 16;
    while (t.BZ > 4 && G.N2 * t.BZ > rc * 256) t.BZ /= 2;
    if (G.N1 * t.BY > rc * 256 || G.N2 * t.BZ > rc * 256)
      throw ArgFail{RISM3D_ERR_ARG, "grid too large for the tile shapes"};
    // small grids (the coarse problem): smaller batches while a pass would
    // otherwise launch fewer than two CTAs per SM
    const long long want = 2 * 148;
    while (t.RX > 4 && (long long)((G.N1 * G.N2 + t.RX - 1) / t.RX) * m < want) t.RX /= 2;
    while (t.BY > 4 && (long long)((G.Nh + t.BY - 1) / t.BY) * G.N2 * m < want) t.BY /= 2;
    while (t.BZ > 4 && (long long)((G.Nh + t.BZ - 1) / t.BZ) * G.N1 < want) t.BZ /= 2;
    // the z tile holds every field's columns: at most 200 KB of shared memory
    const size_t cs = pr == 0 ? sizeof(double2) : sizeof(float2);
    while (t.BZ > 4 && cs * (size_t)G.N2 * (size_t)(m * t.BZ + 1) > 200 * 1024) t.BZ /= 2;
  }
  // FFT plans and twiddles
  const int lens[3] = {G.M, G.N1, G.N2};
  for (int a = 0; a < 3; ++a) {
    std::vector<double2> t64;
    std::vector<float2> t32;
    twiddles(lens[a], t64, t32);
    c->tw64[a] = dalloc<double2>(lens[a]);
    c->tw32[a] = dalloc<float2>(lens[a]);
    CK(cudaMemcpy(c->tw64[a], t64.data(), sizeof(double2) * lens[a], cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->tw32[a], t32.data(), sizeof(float2) * lens[a], cudaMemcpyHostToDevice));
  }
  c->px64 = make_plan(G.M); c->px64.tw = c->tw64[0];
  c->py64 = make_plan(G.N1); c->py64.tw = c->tw64[1];
  c->pz64 = make_plan(G.N2); c->pz64.tw = c->tw64[2];
  c->px32 = c->px64; c->px32.tw = c->tw32[0];
  c->py32 = c->py64; c->py32.tw = c->tw32[1];
  c->pz32 = c->pz64; c->pz32.tw = c->tw32[2];
  {
    std::vector<double2> t64;
    std::vector<float2> t32;
    twiddles(G.N0, t64, t32);  // post twiddles exp(-2 pi i k / N0), k in [0, M]
    c->post64 = dalloc<double2>(G.Nh);
    c->post32 = dalloc<float2>(G.Nh);
    CK(cudaMemcpy(c->post64, t64.data(), sizeof(double2) * G.Nh, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->post32, t32.data(), sizeof(float2) * G.Nh, cudaMemcpyHostToDevice));
  }
}

// The complex work buffer, the reduction partials and the wait-error flag.
void init_work(rism3d_ctx *c) {
  const Geo &G = c->g;
  c->W = dalloc<double2>((size_t)G.m * G.Nc);
  // reduction blocks: about four 16-byte loads per thread, at most 4 per SM
  c->red_blocks = (int)std::min<long long>(592, std::max<long long>(8, (c->nvec / 4 + 1023) / 1024));
  c->dpart = dalloc<double>((size_t)c->red_blocks * (kVecMax + 1) + 64);
  c->dres = dalloc<double>(4 * kVecMax);
  const int rows = G.N1 * G.N2;
  // partials for the smallest x batch the tile autotuner may pick
  const int rxmin = std::min(std::min(c->tiles[0].RX, c->tiles[1].RX), 4);
  c->npart = dalloc<NormPartial>((size_t)((rows + rxmin - 1) / rxmin) * G.m);
  c->d_err = dalloc<int>(1);
  CK(cudaMemset(c->d_err, 0, sizeof(int)));
}

// Shared-memory opt-in: a kernel may use the device's per-block opt-in limit
// minus its own static shared memory, which must cover `need` bytes.
void allow_smem(const void *fn, size_t need) {
  int dev = 0, optin = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  CK(cudaFuncGetAttributes(&fa, fn));
  const int dyn = optin - (int)fa.sharedSizeBytes;
  if ((size_t)dyn < need) throw ArgFail{RISM3D_ERR_ARG, "tile exceeds shared memory"};
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
}

// Largest dynamic shared memory of the runtime-length passes.
size_t generic_smem(rism3d_ctx *c) {
  size_t need = 0;
  for (size_t b : {xsmem<double>(c), ysmem<double>(c), zsmem<double>(c), xsmem<float>(c), ysmem<float>(c),
                   zsmem<float>(c)})
    need = std::max(need, b);
  return need;
}

// Opt-in for the runtime-length x and y passes (every context uses them).
void allow_xy(size_t need) {
  allow_smem((const void *)k_xfwd<double, MODE_F>, need);
  allow_smem((const void *)k_xfwd<double, MODE_J>, need);
  allow_smem((const void *)k_xfwd<float, MODE_F>, need);
  allow_smem((const void *)k_xfwd<float, MODE_J>, need);
  allow_smem((const void *)k_xinv<double>, need);
  allow_smem((const void *)k_xinv<float>, need);
  allow_smem((const void *)k_xfwd<double, MODE_FWD>, need);
#define OPTIN_Y(T)                                          \
  allow_smem((const void *)k_y<T, false, 16>, need);        \
  allow_smem((const void *)k_y<T, true, 16>, need);         \
  allow_smem((const void *)k_y<T, false, 8>, need);         \
  allow_smem((const void *)k_y<T, true, 8>, need);          \
  allow_smem((const void *)k_y<T, false, 4>, need);         \
  allow_smem((const void *)k_y<T, true, 4>, need);
  OPTIN_Y(double)
  OPTIN_Y(float)
#undef OPTIN_Y
}

// chi3 (optional): chi - 1 on the k grid, packed pairs of complex
// [m(m+1)/2][N2][N1][N0/2+1] (the --solvent-3d kernel); then chi is unused,
// the long-range term takes the no-renorm form and the passes are the
// runtime-length ones without the two-grid preconditioner.
int create_impl(const rism3d_problem *pd, int m, const rism3d_site *solvent, int n, const rism3d_site *solute,
                const double *chi, const double *chi3, rism3d_ctx **out) {
  if (!pd || !solvent || (!solute && n > 0) || (!chi && !chi3) || !out) throw ArgFail{RISM3D_ERR_ARG, "null argument"};
  if (m < 1 || m > kMaxSites) throw ArgFail{RISM3D_ERR_ARG, "solvent sites must be 1..6"};
  if (n < 0) throw ArgFail{RISM3D_ERR_ARG, "negative solute size"};
  check_grid(pd);
  if (!chi3 && (pd->nrad < 4 || !(pd->rmax > 0))) throw ArgFail{RISM3D_ERR_ARG, "bad radial grid"};
  auto c = new rism3d_ctx();
  try {
    c->pd = *pd;
    if (chi3) {
      c->pd.renorm = 0;
      c->pd.coarse_h = 0;
    }
    pd = &c->pd;
    c->m = m;
    c->n = n;
    c->solvent.assign(solvent, solvent + m);
    c->solute.assign(solute, solute + n);
    const double pi = 3.14159265358979323846;
    if (!chi3) {
      // |k| of every grid point must fall inside the chi table (interp
      // assert, bgy3d-vec.c:30-31); checked before any device work
      const double dk[3] = {2 * pi / pd->L[0], 2 * pi / pd->L[1], 2 * pi / pd->L[2]};
      const double kmax = std::sqrt(std::pow(pd->N[0] / 2 * dk[0], 2) + std::pow(pd->N[1] / 2 * dk[1], 2) +
                                    std::pow(pd->N[2] / 2 * dk[2], 2));
      if ((int)(kmax / (pi / pd->rmax) - 0.5 + 0.5) >= pd->nrad) throw ArgFail{RISM3D_ERR_TABLE, "chi table too short"};
    }
    init_grid(c, m);
    const Geo &G = c->g;
    for (int i = 0; i < m; ++i) c->charge.push_back(solvent[i].charge);

    const int npair = m * (m + 1) / 2;
    if (chi3) {
      // chi - 1 on the k grid into the padded W layout [pair][N2][N1][Nhp]
      const size_t rows = (size_t)npair * G.N2 * G.N1;
      c->chi3_64 = dalloc<double2>((size_t)npair * G.Nc);
      c->chi3_32 = dalloc<float2>((size_t)npair * G.Nc);
      CK(cudaMemset(c->chi3_64, 0, sizeof(double2) * (size_t)npair * G.Nc));
      CK(cudaMemset(c->chi3_32, 0, sizeof(float2) * (size_t)npair * G.Nc));
      CK(cudaMemcpy2D(c->chi3_64, sizeof(double2) * G.Nhp, chi3, sizeof(double2) * G.Nh, sizeof(double2) * G.Nh,
                      rows, cudaMemcpyHostToDevice));
      std::vector<float2> h32(rows * G.Nh);
      for (size_t q = 0; q < h32.size(); ++q) h32[q] = make_float2((float)chi3[2 * q], (float)chi3[2 * q + 1]);
      CK(cudaMemcpy2D(c->chi3_32, sizeof(float2) * G.Nhp, h32.data(), sizeof(float2) * G.Nh, sizeof(float2) * G.Nh,
                      rows, cudaMemcpyHostToDevice));
    } else {
      // radial tables: chi - delta (solvent_kernel_rism, hnc3d.c:1548-1556) and
      // beta/eps0 s_i (rism_solvent_renorm, rism.f90:141-208)
      const int nrad = pd->nrad;
      std::vector<double2> chi64((size_t)npair * nrad), s64((size_t)m * nrad);
      std::vector<double> tab(nrad);
      std::vector<double2> pr;
      for (int i = 0; i < m; ++i)
        for (int j = 0; j <= i; ++j) {
          for (int k = 0; k < nrad; ++k) tab[k] = chi[((size_t)i * m + j) * nrad + k] - (i == j ? 1.0 : 0.0);
          interp_pairs(tab.data(), nrad, pr);
          std::copy(pr.begin(), pr.end(), chi64.begin() + (size_t)(i * (i + 1) / 2 + j) * nrad);
        }
      const double dk = pi / pd->rmax;
      for (int i = 0; i < m; ++i) {
        std::vector<double> x(nrad, 0.0);
        for (int j = 0; j < m; ++j)
          for (int k = 0; k < nrad; ++k) x[k] = x[k] + chi[((size_t)j * m + i) * nrad + k] * solvent[j].charge;
        for (int k = 0; k < nrad; ++k) {
          const double kk = (2 * (k + 1) - 1) * dk / 2;
          const double v = kk == 0.0 ? 0.0 : 4 * pi * std::exp(-kk * kk / (4 * kG * kG)) / (kk * kk);
          tab[k] = pd->beta * kEps0Inv * (x[k] * v);
        }
        interp_pairs(tab.data(), nrad, pr);
        std::copy(pr.begin(), pr.end(), s64.begin() + (size_t)i * nrad);
      }
      std::vector<float2> chi32(chi64.size()), s32(s64.size());
      for (size_t i = 0; i < chi64.size(); ++i) chi32[i] = make_float2((float)chi64[i].x, (float)chi64[i].y);
      for (size_t i = 0; i < s64.size(); ++i) s32[i] = make_float2((float)s64[i].x, (float)s64[i].y);
      c->chi64 = dalloc<double2>(chi64.size());
      c->chi32 = dalloc<float2>(chi32.size());
      c->s64 = dalloc<double2>(s64.size());
      c->s32 = dalloc<float2>(s32.size());
      CK(cudaMemcpy(c->chi64, chi64.data(), sizeof(double2) * chi64.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(c->chi32, chi32.data(), sizeof(float2) * chi32.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(c->s64, s64.data(), sizeof(double2) * s64.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(c->s32, s32.data(), sizeof(float2) * s32.size(), cudaMemcpyHostToDevice));
    }

    // sites
    std::vector<SiteP> hv(m);
    for (int i = 0; i < m; ++i)
      hv[i] = SiteP{solvent[i].x[0], solvent[i].x[1], solvent[i].x[2], solvent[i].sigma, solvent[i].epsilon,
                    solvent[i].charge};
    c->d_solvent = dalloc<SiteP>(m);
    CK(cudaMemcpy(c->d_solvent, hv.data(), sizeof(SiteP) * m, cudaMemcpyHostToDevice));
    c->d_charge = dalloc<double>(m);
    CK(cudaMemcpy(c->d_charge, c->charge.data(), sizeof(double) * m, cudaMemcpyHostToDevice));

    // fields of the solute
    c->v64 = dalloc<double>(c->nvec);
    c->v32 = dalloc<float>(c->nvec);
    c->L64 = dalloc<double2>((size_t)G.Nc);
    c->L32 = dalloc<float2>((size_t)G.Nc);
    bind_solute(c, n, solute);
    init_work(c);
    // shape-specialised passes (TMA tiles) for the lengths they are built for;
    // RISM3D_GENERIC_PASSES=1 selects the runtime-length passes everywhere
    const char *gen = std::getenv("RISM3D_GENERIC_PASSES");
    if (static_len_x(G.M) && static_len_yz(G.N1) && static_len_yz(G.N2) && m <= 3 && !chi3 &&
        !(gen && gen[0] == '1')) {
      for (int pr = 0; pr < 2; ++pr) {
        const int B = pr == 0 ? static_B<double>() : static_B<float>();
        make_tmap(c, &c->tmy[pr], pr == 0, B, G.N1, 1);
        make_tmap(c, &c->tmz[pr], pr == 0, c->zb[pr], 1, G.N2);
        c->stat[pr] = true;
      }
    }
    size_t need = generic_smem(c);
    allow_xy(need);
    auto allow = [&](const void *fn) { allow_smem(fn, need); };
    allow((const void *)k_z<double, MODE_FWD, 16>);  // forward transform of the gradient
    allow((const void *)k_z<double, MODE_FWD, 8>);
    allow((const void *)k_z<double, MODE_FWD, 4>);
#define OPTIN_Z(T)                                   \
  allow((const void *)k_z<T, MODE_F, 16>);           \
  allow((const void *)k_z<T, MODE_J, 16>);           \
  allow((const void *)k_z<T, MODE_F, 8>);            \
  allow((const void *)k_z<T, MODE_J, 8>);            \
  allow((const void *)k_z<T, MODE_F, 4>);            \
  allow((const void *)k_z<T, MODE_J, 4>);
    OPTIN_Z(double)
    OPTIN_Z(float)
#undef OPTIN_Z
    if (c->stat[0]) {
      need = std::max({xs_smem<double, 256>(), ys_smem<double, 512>(), zsp_smem<double, 512>(m),
                       zsp_smem<float, 512>(m), zs_smem<double, 512>(m),
                       xs_smem<float, 256>(), ys_smem<float, 512>(), zs_smem<float, 512>(m)});
#define OPTIN_S(T)                                               \
  allow((const void *)k_xfwd_s<T, MODE_F, 24, kStaticRX>);       \
  allow((const void *)k_xfwd_s<T, MODE_J, 24, kStaticRX>);       \
  allow((const void *)k_xinv_s<T, 24, kStaticRX>);               \
  allow((const void *)k_xfwd_s<T, MODE_F, 32, kStaticRX>);       \
  allow((const void *)k_xfwd_s<T, MODE_J, 32, kStaticRX>);       \
  allow((const void *)k_xinv_s<T, 32, kStaticRX>);               \
  allow((const void *)k_xfwd_s<T, MODE_F, 36, kStaticRX>);       \
  allow((const void *)k_xfwd_s<T, MODE_J, 36, kStaticRX>);       \
  allow((const void *)k_xinv_s<T, 36, kStaticRX>);               \
  allow((const void *)k_xfwd_s<T, MODE_F, 48, kStaticRX>);       \
  allow((const void *)k_xfwd_s<T, MODE_J, 48, kStaticRX>);       \
  allow((const void *)k_xinv_s<T, 48, kStaticRX>);               \
  allow((const void *)k_xfwd_s<T, MODE_F, 64, kStaticRX>);       \
  allow((const void *)k_xfwd_s<T, MODE_J, 64, kStaticRX>);       \
  allow((const void *)k_xinv_s<T, 64, kStaticRX>);               \
  allow((const void *)k_xfwd_s<T, MODE_F, 72, kStaticRX>);       \
  allow((const void *)k_xfwd_s<T, MODE_J, 72, kStaticRX>);       \
  allow((const void *)k_xinv_s<T, 72, kStaticRX>);               \
  allow((const void *)k_xfwd_s<T, MODE_F, 96, kStaticRX>);       \
  allow((const void *)k_xfwd_s<T, MODE_J, 96, kStaticRX>);       \
  allow((const void *)k_xinv_s<T, 96, kStaticRX>);               \
  allow((const void *)k_xfwd_s<T, MODE_F, 128, kStaticRX>);      \
  allow((const void *)k_xfwd_s<T, MODE_J, 128, kStaticRX>);      \
  allow((const void *)k_xinv_s<T, 128, kStaticRX>);              \
  allow((const void *)k_xfwd_s<T, MODE_F, 256, kStaticRX>);      \
  allow((const void *)k_xfwd_s<T, MODE_J, 256, kStaticRX>);      \
  allow((const void *)k_xinv_s<T, 256, kStaticRX>);              \
  allow((const void *)k_y_s<T, false, 512, static_B<T>()>);      \
  allow((const void *)k_y_s<T, true, 512, static_B<T>()>);       \
  allow((const void *)k_z_s<T, MODE_F, 512, static_Bz<T>(), 3>); \
  allow((const void *)k_z_s<T, MODE_J, 512, static_Bz<T>(), 3>); \
  allow((const void *)k_z_s<T, MODE_F, 512, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_J, 512, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_sp<T, MODE_F, 512, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_J, 512, static_Bz<T>(), 3>);   \
  allow((const void *)k_y_s<T, false, 48, static_B<T>()>);       \
  allow((const void *)k_y_s<T, true, 48, static_B<T>()>);        \
  allow((const void *)k_z_s<T, MODE_F, 48, static_Bz<T>(), 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 48, static_Bz<T>(), 3>);  \
  allow((const void *)k_y_s<T, false, 64, static_B<T>()>);       \
  allow((const void *)k_y_s<T, true, 64, static_B<T>()>);        \
  allow((const void *)k_z_s<T, MODE_F, 64, static_Bz<T>(), 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 64, static_Bz<T>(), 3>);  \
  allow((const void *)k_y_s<T, false, 72, static_B<T>()>);       \
  allow((const void *)k_y_s<T, true, 72, static_B<T>()>);        \
  allow((const void *)k_z_s<T, MODE_F, 72, static_Bz<T>(), 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 72, static_Bz<T>(), 3>);  \
  allow((const void *)k_y_s<T, false, 96, static_B<T>()>);       \
  allow((const void *)k_y_s<T, true, 96, static_B<T>()>);        \
  allow((const void *)k_z_s<T, MODE_F, 96, static_Bz<T>(), 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 96, static_Bz<T>(), 3>);  \
  allow((const void *)k_y_s<T, false, 128, static_B<T>()>);      \
  allow((const void *)k_y_s<T, true, 128, static_B<T>()>);       \
  allow((const void *)k_z_s<T, MODE_F, 128, static_Bz<T>(), 3>); \
  allow((const void *)k_z_s<T, MODE_J, 128, static_Bz<T>(), 3>); \
  allow((const void *)k_y_s<T, false, 144, static_B<T>()>);      \
  allow((const void *)k_y_s<T, true, 144, static_B<T>()>);       \
  allow((const void *)k_z_s<T, MODE_F, 144, static_Bz<T>(), 3>); \
  allow((const void *)k_z_s<T, MODE_J, 144, static_Bz<T>(), 3>); \
  allow((const void *)k_y_s<T, false, 192, static_B<T>()>);      \
  allow((const void *)k_y_s<T, true, 192, static_B<T>()>);       \
  allow((const void *)k_z_s<T, MODE_F, 192, static_Bz<T>(), 3>); \
  allow((const void *)k_z_s<T, MODE_J, 192, static_Bz<T>(), 3>); \
  allow((const void *)k_y_s<T, false, 256, static_B<T>()>);      \
  allow((const void *)k_y_s<T, true, 256, static_B<T>()>);       \
  allow((const void *)k_z_s<T, MODE_F, 256, static_Bz<T>(), 3>); \
  allow((const void *)k_z_s<T, MODE_J, 256, static_Bz<T>(), 3>); \
  allow((const void *)k_z_s<T, MODE_F, 48, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 48, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_F, 64, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 64, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_F, 72, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 72, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_F, 96, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_J, 96, static_Bz<T>() / 2, 3>);  \
  allow((const void *)k_z_s<T, MODE_F, 128, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_J, 128, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_F, 144, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_J, 144, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_F, 192, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_J, 192, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_F, 256, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_s<T, MODE_J, 256, static_Bz<T>() / 2, 3>); \
  allow((const void *)k_z_sp<T, MODE_F, 48, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_J, 48, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_F, 64, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_J, 64, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_F, 72, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_J, 72, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_F, 96, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_J, 96, static_Bz<T>(), 3>);    \
  allow((const void *)k_z_sp<T, MODE_F, 128, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_J, 128, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_F, 144, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_J, 144, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_F, 192, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_J, 192, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_F, 256, static_Bz<T>(), 3>);   \
  allow((const void *)k_z_sp<T, MODE_J, 256, static_Bz<T>(), 3>);
      OPTIN_S(double)
      OPTIN_S(float)
#undef OPTIN_S
    }
    autotune(c);
    // two-grid preconditioner: a copy of the problem on a coarse grid.  The
    // spacing coarse_h is taken when its grid has at most half the fine
    // points along every axis (a coarse solve costs ~12 coarse J.v per fine
    // iteration); otherwise 1 A (or coarse_h if coarser), when that grid is
    // still coarser than the fine one; otherwise the preconditioner is off.
    if (pd->coarse_h > 0 && pd->solver != RISM3D_PICARD && pd->solver != RISM3D_JAGER) {
      auto grid_for = [&](double h, int *nc) {
        bool half = true;
        for (int a = 0; a < 3; ++a) {
          int nn = std::max(8, (int)std::ceil(pd->L[a] / h - 1e-9));
          while (!(is_2a3b(nn) && nn % 2 == 0)) ++nn;
          nc[a] = nn;
          if (2 * nn > pd->N[a]) half = false;
        }
        return half;
      };
      int nc[3];
      bool coarser = true;
      if (!grid_for(pd->coarse_h, nc)) {
        grid_for(std::max(pd->coarse_h, 1.0), nc);
        for (int a = 0; a < 3; ++a)
          if (nc[a] >= pd->N[a]) coarser = false;
      }
      if (coarser) {
        rism3d_problem pc = *pd;
        for (int a = 0; a < 3; ++a) pc.N[a] = nc[a];
        pc.coarse_h = 0;
        pc.verbosity = 0;
        create_impl(&pc, m, solvent, n, solute, chi, nullptr, &c->coarse);
        for (int a = 0; a < 3; ++a) {
          const int nf = pd->N[a], ncs = nc[a];
          c->Nc[a] = ncs;
          std::vector<float> R((size_t)ncs * nf), Rt((size_t)nf * ncs), P((size_t)nf * ncs), Pt((size_t)ncs * nf);
          // s(x) = sum_{|k| <= K} w_k cos(2 pi k x), K = ncs / 2, w_{+-K} = 1/2:
          // the Dirichlet kernel sin((2K - 1) pi x) / sin(pi x) of |k| < K
          // plus cos(2 pi K x); x = i/ncs - j/nf = (i nf - j ncs) / (ncs nf)
          const int K = ncs / 2;
          const long long den = (long long)ncs * nf;
          for (int i = 0; i < ncs; ++i)
            for (int j = 0; j < nf; ++j) {
              long long q = ((long long)i * nf - (long long)j * ncs) % den;
              if (q < 0) q += den;
              const double x = (double)q / (double)den;  // in [0, 1)
              const double sx = std::sin(pi * x);
              double s = std::fabs(sx) < 1e-12 ? (double)(2 * K - 1) : std::sin((2 * K - 1) * pi * x) / sx;
              s += std::cos(2.0 * pi * K * x);
              R[(size_t)i * nf + j] = Rt[(size_t)j * ncs + i] = (float)(s / nf);
              P[(size_t)j * ncs + i] = Pt[(size_t)i * nf + j] = (float)(s / ncs);
            }
          auto up = [&](const std::vector<float> &h) {
            float *dptr = dalloc<float>(h.size());
            CK(cudaMemcpy(dptr, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
            return dptr;
          };
          c->tR[a] = up(R);
          c->tRt[a] = up(Rt);
          c->tP[a] = up(P);
          c->tPt[a] = up(Pt);
        }
        {  // x-axis FFT-transfer tables, K = Nc0 / 2: C [K+1][Nc0], D [Nc0][K+1]
          const int ncx = c->Nc[0], K = ncx / 2, n0 = pd->N[0];
          std::vector<float2> Ct((size_t)(K + 1) * ncx), Dt((size_t)(K + 1) * ncx);
          for (int k = 0; k <= K; ++k)
            for (int i = 0; i < ncx; ++i) {
              const double ph = 2.0 * pi * ((long long)k * i % ncx) / ncx;
              const double ck = (k == 0 || 2 * k == ncx) ? 1.0 : 2.0;
              const double fk = (2 * k == ncx) ? 0.5 / ncx : 1.0 / ncx;
              Ct[(size_t)k * ncx + i] = make_float2((float)(ck * std::cos(ph) / n0), (float)(ck * std::sin(ph) / n0));
              Dt[(size_t)i * (K + 1) + k] = make_float2((float)(fk * std::cos(ph)), (float)(-fk * std::sin(ph)));
            }
          c->tC = dalloc<float2>(Ct.size());
          c->tD = dalloc<float2>(Dt.size());
          CK(cudaMemcpy(c->tC, Ct.data(), sizeof(float2) * Ct.size(), cudaMemcpyHostToDevice));
          CK(cudaMemcpy(c->tD, Dt.data(), sizeof(float2) * Dt.size(), cudaMemcpyHostToDevice));
        }
        allow_smem((const void *)tg::k_transfer_axis_j<32>, sizeof(float) * tg::kAxMaxIn * 32);
        allow_smem((const void *)tg::k_transfer_axis_j<16>, sizeof(float) * tg::kAxMaxIn * 16);
        c->tA = dalloc<float>((size_t)m * G.N2 * G.N1 * c->Nc[0]);
        c->tB = dalloc<float>((size_t)m * G.N2 * c->Nc[1] * c->Nc[0]);
        c->tc_r = dalloc<float>(c->coarse->nvec);
        c->tc_y = dalloc<float>(c->coarse->nvec);
      }
    }
  } catch (...) {
    delete c;
    throw;
  }
  *out = c;
  return RISM3D_OK;
}

// A pure-solvent context (hnc3d_solvent_solve, hnc3d.c:803-1073): the
// m(m+1)/2 site-site pair fields run through the residual / Jacobian passes
// with the molecular OZ z pass.  FP64, Newton-GMRES, no preconditioner.
int solvent_create_impl(const rism3d_problem *pd, int ms, const rism3d_site *solvent, rism3d_ctx **out) {
  if (!pd || !solvent || !out) throw ArgFail{RISM3D_ERR_ARG, "null argument"};
  if (ms < 1 || ms > kMaxSolventSites) throw ArgFail{RISM3D_ERR_ARG, "pure-solvent sites must be 1..4"};
  check_grid(pd);
  // omega_intra takes k r from L[0] and asserts a cubic box (bgy3d-pure.c:247-250)
  if (pd->L[1] != pd->L[0] || pd->L[2] != pd->L[0]) throw ArgFail{RISM3D_ERR_ARG, "the pure solvent needs a cubic box"};
  if (pd->closure == RISM3D_PY) throw ArgFail{RISM3D_ERR_UNSUPPORTED, "PY has no closure differential"};
  auto c = new rism3d_ctx();
  try {
    c->pd = *pd;
    c->pd.renorm = 0;
    c->pd.coarse_h = 0;
    c->pd.precision = RISM3D_FP64;
    const int np = ms * (ms + 1) / 2;
    c->pure = ms;
    c->m = np;
    c->n = 0;
    c->solvent.assign(solvent, solvent + ms);
    init_grid(c, np);
    const Geo &G = c->g;
    const double pi = 3.14159265358979323846;
    std::vector<PairP> hp;
    for (int i = 0; i < ms; ++i)
      for (int j = 0; j <= i; ++j) {
        const rism3d_site &a = solvent[i], &b = solvent[j];
        const double q2 = a.charge * b.charge;
        hp.push_back(PairP{0.5 * (a.sigma + b.sigma), std::sqrt(a.epsilon * b.epsilon), q2});
        const double dx = a.x[0] - b.x[0], dy = a.x[1] - b.x[1], dz = a.x[2] - b.x[2];
        c->pq2.push_back(q2);
        c->pwr.push_back(2.0 * pi * std::sqrt(dx * dx + dy * dy + dz * dz) / pd->L[0]);
      }
    PairP *dp = dalloc<PairP>(np);
    CK(cudaMemcpy(dp, hp.data(), sizeof(PairP) * np, cudaMemcpyHostToDevice));
    c->v64 = dalloc<double>(c->nvec);
    const double h0 = pd->L[0] / pd->N[0], h1 = pd->L[1] / pd->N[1], h2 = pd->L[2] / pd->N[2];
    k_pair_field<<<(unsigned)((G.Nr + 255) / 256), 256, 0, c->stream>>>(G, h0, h1, h2, pd->L[0], pd->L[1], pd->L[2],
                                                                        dp, c->v64);
    CKL();
    dfree(dp);
    c->ck = dalloc<double2>((size_t)np * G.Nc);
    CK(cudaMemsetAsync(c->ck, 0, sizeof(double2) * (size_t)np * G.Nc, c->stream));
    init_work(c);
    const size_t need = generic_smem(c);
    allow_xy(need);
    allow_smem((const void *)k_z<double, MODE_FWD, 16>, need);
    allow_smem((const void *)k_z<double, MODE_FWD, 8>, need);
    allow_smem((const void *)k_z<double, MODE_FWD, 4>, need);
    switch (ms) {
      case 1: allow_oz<1>(need); break;
      case 2: allow_oz<2>(need); break;
      case 3: allow_oz<3>(need); break;
      default: allow_oz<4>(need); break;
    }
    autotune(c);
    CK(cudaStreamSynchronize(c->stream));
  } catch (...) {
    delete c;
    throw;
  }
  *out = c;
  return RISM3D_OK;
}

// The real-space long-range correlation c_L = -beta v_L of every pair by an
// inverse transform of its k-space form (hnc3d.c:990-1003), into out.
void long_range_field(rism3d_ctx *c, double *out) {
  {
    TimeScope ts(c, TK_Z, 0);
    switch (c->pure) {
      case 1: launch_oz_ms<MODE_VL, 1>(c); break;
      case 2: launch_oz_ms<MODE_VL, 2>(c); break;
      case 3: launch_oz_ms<MODE_VL, 3>(c); break;
      default: launch_oz_ms<MODE_VL, 4>(c); break;
    }
  }
  launch_y<double, true>(c);
  TimeScope ts(c, TK_XINV, 0);
  const int RX = c->tl<double>().RX;
  dim3 gx((c->g.N1 * c->g.N2 + RX - 1) / RX, c->m);
  k_xinv<double><<<gx, 256, xsmem<double>(c), c->stream>>>(c->g, c->plan<double>(0), RX, c->work<double>(), out, out,
                                                          1.0 / (double)c->g.Nr, 0.0, postw<double>(c), c->npart);
  CKL();
}

// Tabulates the 1D RISM t(r) of the pure solvent on the upscaled radial grid
// (rmax = 2 max(L), nrad = 16 max(N): upscale, hnc3d.c:776-787) on the 3D
// grid as the initial guess (hnc3d.c:824-851).
void solvent_guess(rism3d_ctx *c, double *T) {
  const rism3d_problem &pd = c->pd;
  const int ms = c->pure;
  rism3d_problem up = pd;
  up.rmax = 4 * std::max(std::max(pd.L[0], pd.L[1]), pd.L[2]) / 2;
  up.nrad = 16 * std::max(std::max(pd.N[0], pd.N[1]), pd.N[2]);
  up.norm_tol = std::max(pd.norm_tol, 1e-10);
  const int nrad = up.nrad;
  std::vector<double> chi((size_t)ms * ms * nrad), t((size_t)ms * ms * nrad, 0.0);
  const int rc = rism1d_solvent_chi(&up, 0.0, ms, c->solvent.data(), chi.data(), t.data(), nullptr);
  if (rc != RISM3D_OK) throw CudaFail{rc};
  std::vector<double2> tab, pr;
  for (int i = 0; i < ms; ++i)
    for (int j = 0; j <= i; ++j) {
      interp_pairs(t.data() + ((size_t)i * ms + j) * nrad, nrad, pr);
      tab.insert(tab.end(), pr.begin(), pr.end());
    }
  double2 *dt = dalloc<double2>(tab.size());
  CK(cudaMemcpy(dt, tab.data(), sizeof(double2) * tab.size(), cudaMemcpyHostToDevice));
  const Geo &G = c->g;
  const double h0 = pd.L[0] / pd.N[0], h1 = pd.L[1] / pd.N[1], h2 = pd.L[2] / pd.N[2];
  k_rtab<<<(unsigned)((G.Nr + 255) / 256), 256, 0, c->stream>>>(G, h0, h1, h2, pd.L[0], pd.L[1], pd.L[2], dt, nrad,
                                                                up.rmax / nrad, T);
  CKL();
  dfree(dt);
}

template <int MS> void chi_out_launch(rism3d_ctx *c, double2 *out) {
  PureParams<MS> pp{};
  pp.rho = c->pd.rho;
  pp.beta = c->pd.beta;
  pp.h3 = c->h3;
  for (int p = 0; p < PureParams<MS>::NP; ++p) {
    pp.q2[p] = c->pq2[p];
    pp.wr[p] = c->pwr[p];
  }
  k_chi_out<MS><<<vec_grid((long long)c->g.Nh * c->g.N1 * c->g.N2), 256, 0, c->stream>>>(c->g, c->work<double>(),
                                                                                           pp, out);
  CKL();
}

// Newton-GMRES on the pair fields from T (device, in/out), then the
// observables, chi - 1 on the k grid and g (host outputs, each optional).
int solvent_solve_impl(rism3d_ctx *c, double *T, double *chi_out, double *g_out, rism3d_solvent_result *res) {
  const rism3d_problem &pd = c->pd;
  *res = rism3d_solvent_result{};
  c->f_evals = c->jv_evals = 0;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c->stream));
  const int restart = pd.krylov_restart > 0 ? std::min(pd.krylov_restart, 200) : 30;
  NewtonOut o = newton<double, double>(c, T, pd.norm_tol, pd.max_iter, 1e-3, restart);
  const Geo &G = c->g;
  const long long nv = c->nvec;
  double *cl = dalloc<double>(nv), *h = dalloc<double>(nv);
  double *g = g_out ? dalloc<double>(nv) : nullptr;
  long_range_field(c, cl);
  const int rb = (int)std::min<long long>(2 * 148, (G.Nr + 255) / 256);
  double *part = dalloc<double>((size_t)rb * 5);
  k_solvent_obs<<<rb, 256, 0, c->stream>>>(G, c->pure, T, c->v64, cl, pd.beta, pd.closure, h, g, part);
  CKL();
  std::vector<double> hp((size_t)rb * 5);
  CK(cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, c->stream));
  if (chi_out) {
    fwd3d(c, h);
    const long long nk = (long long)G.Nh * G.N1 * G.N2;
    double2 *dchi = dalloc<double2>((size_t)c->m * nk);
    switch (c->pure) {
      case 1: chi_out_launch<1>(c, dchi); break;
      case 2: chi_out_launch<2>(c, dchi); break;
      case 3: chi_out_launch<3>(c, dchi); break;
      default: chi_out_launch<4>(c, dchi); break;
    }
    CK(cudaMemcpyAsync(chi_out, dchi, sizeof(double2) * (size_t)c->m * nk, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    dfree(dchi);
  }
  if (g_out) CK(cudaMemcpyAsync(g_out, g, sizeof(double) * nv, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dfree(cl);
  dfree(h);
  dfree(g);
  dfree(part);
  double a[5] = {0, 0, 0, 0, 0};
  for (int b = 0; b < rb; ++b)
    for (int k = 0; k < 5; ++k) a[k] += hp[(size_t)b * 5 + k];
  // mu = rho h^3 sum / beta (chempot, hnc3d.c:604-623); kappa and a from
  // rho c(k=0) = rho h^3 sum c (print_kappa, hnc3d.c:738-760)
  const double f = pd.rho * c->h3 / pd.beta;
  res->mu = a[0] * f;
  res->mu_hnc = a[1] * f;
  res->mu_kh = a[2] * f;
  res->mu_gf = a[3] * f;
  const double c0 = a[4] * (pd.rho * c->h3);
  res->a = c0 / 2 / pd.beta;
  res->kappa = pd.beta / (1 - c0) / pd.rho;
  res->resid_inf = o.rinf;
  res->resid_2 = o.r2;
  res->newton_iters = o.iters;
  res->f_evals = c->f_evals;
  res->jv_evals = c->jv_evals;
  res->seconds = ms * 1e-3;
  res->status = o.nan ? RISM3D_ERR_NAN : (o.converged ? RISM3D_OK : RISM3D_ERR_NOT_CONVERGED);
  return res->status;
}

// Moments of shift + scale * v over `nf` fields into out[nf][13] (q, d[3],
// Q[3][3]) with the h^3, h_a, h_a h_b scales of bgy3d_moments.
void moments_of(rism3d_ctx *c, const double *v, int nf, double shift, double scale, double *out) {
  const Geo &G = c->g;
  const int rb = (int)std::min<long long>(2 * 148, (G.Nr + 255) / 256);
  double *part = dalloc<double>((size_t)rb * nf * 10);
  k_moments<<<dim3(rb, nf), 256, 0, c->stream>>>(G, v, nf, shift, scale, part);
  CKL();
  std::vector<double> hp((size_t)rb * nf * 10);
  CK(cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  dfree(part);
  const double h[3] = {c->pd.L[0] / c->pd.N[0], c->pd.L[1] / c->pd.N[1], c->pd.L[2] / c->pd.N[2]};
  const double dV = c->h3;
  for (int f = 0; f < nf; ++f) {
    double a[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < rb; ++b)
      for (int k = 0; k < 10; ++k) a[k] += hp[((size_t)f * rb + b) * 10 + k];
    double *o = out + (size_t)f * 13;
    o[0] = dV * a[0];
    for (int d = 0; d < 3; ++d) o[1 + d] = dV * h[d] * a[1 + d];
    const int diag[3] = {4, 5, 6};
    for (int d = 0; d < 3; ++d) o[4 + 4 * d] = dV * h[d] * h[d] * a[diag[d]];
    o[4 + 1] = o[4 + 3] = dV * h[0] * h[1] * a[7];
    o[4 + 5] = o[4 + 7] = dV * h[1] * h[2] * a[8];
    o[4 + 2] = o[4 + 6] = dV * h[0] * h[2] * a[9];
  }
}

int info_impl(rism3d_ctx *c, const double *T, rism3d_info_result *res, double *site_potential) {
  const rism3d_problem &pd = c->pd;
  const Geo &G = c->g;
  *res = rism3d_info_result{};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c->stream));
  const double h[3] = {pd.L[0] / pd.N[0], pd.L[1] / pd.N[1], pd.L[2] / pd.N[2]};
  const unsigned nb = (unsigned)((G.Nr + 255) / 256);
  double *A = dalloc<double>(c->nvec), *ru = dalloc<double>(G.Nr), *uc = dalloc<double>(G.Nr);
  double2 *Rv = dalloc<double2>((size_t)G.Nc);
  CK(cudaMemsetAsync(A, 0, sizeof(double) * c->nvec, c->stream));
  double *rv = A;  // field 0 of A: the forward transform takes it from there
  k_densities<<<nb, 256, 0, c->stream>>>(G, c->m, T, c->v64, pd.beta, pd.closure, c->d_charge, pd.rho, h[0], h[1],
                                         h[2], pd.L[0], pd.L[1], pd.L[2], c->n, c->d_solute, rv, ru);
  CKL();
  k_coulomb_long<<<nb, 256, 0, c->stream>>>(G, h[0], h[1], h[2], pd.L[0], pd.L[1], pd.L[2], c->n, c->d_solute, uc);
  CKL();
  double mu[13], mv[13];
  moments_of(c, ru, 1, 0.0, 1.0, mu);
  moments_of(c, rv, 1, 0.0, 1.0, mv);
  const int rb = (int)std::min<long long>(2 * 148, (G.Nr + 255) / 256);
  double *dpart = dalloc<double>(rb);
  k_dot<<<rb, 256, 0, c->stream>>>(G.Nr, uc, rv, dpart);
  CKL();
  std::vector<double> hd(rb);
  CK(cudaMemcpyAsync(hd.data(), dpart, sizeof(double) * rb, cudaMemcpyDeviceToHost, c->stream));
  // spectra: Rv kept aside, Ru left in W
  fwd3d(c, A);
  CK(cudaMemcpyAsync(Rv, c->work<double>(), sizeof(double2) * G.Nc, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(A, ru, sizeof(double) * G.Nr, cudaMemcpyDeviceToDevice, c->stream));
  fwd3d(c, A);
  // points: the solute sites, then the 8 grid nodes around each
  const int n = c->n;
  std::vector<double3> pts;
  std::vector<double> fr(3 * (size_t)n);
  for (int u = 0; u < n; ++u) {
    double y[3];
    for (int d = 0; d < 3; ++d) y[d] = (c->solute[u].x[d] + pd.L[d] / 2) / h[d];
    pts.push_back(make_double3(y[0], y[1], y[2]));
  }
  for (int u = 0; u < n; ++u) {
    const double3 y = pts[u];
    const double fl[3] = {std::floor(y.x), std::floor(y.y), std::floor(y.z)};
    fr[3 * u] = y.x - fl[0];
    fr[3 * u + 1] = y.y - fl[1];
    fr[3 * u + 2] = y.z - fl[2];
    for (int q = 0; q < 8; ++q) pts.push_back(make_double3(fl[0] + (q & 1), fl[1] + ((q >> 1) & 1), fl[2] + (q >> 2)));
  }
  const int npts = (int)pts.size();
  double3 *dpts = dalloc<double3>(std::max(npts, 1));
  if (npts) CK(cudaMemcpyAsync(dpts, pts.data(), sizeof(double3) * npts, cudaMemcpyHostToDevice, c->stream));
  const long long nk = (long long)G.Nh * G.N1 * G.N2;
  const int kb = (int)std::min<long long>(2 * 148, (nk + 255) / 256);
  double *kpart = dalloc<double>((size_t)kb * (npts + 1));
  k_info_kspace<<<dim3(kb, npts + 1), 256, 0, c->stream>>>(G, Rv, c->work<double>(), npts, dpts, kpart);
  CKL();
  std::vector<double> hk((size_t)kb * (npts + 1));
  CK(cudaMemcpyAsync(hk.data(), kpart, sizeof(double) * hk.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (void *p : {(void *)A, (void *)ru, (void *)uc, (void *)Rv, (void *)dpart, (void *)dpts, (void *)kpart}) dfree(p);
  const double Ntot = (double)G.Nr;
  std::vector<double> val(npts + 1, 0.0);
  for (int q = 0; q <= npts; ++q)
    for (int b = 0; b < kb; ++b) val[q] += hk[(size_t)q * kb + b];
  for (int q = 0; q < npts; ++q) val[q] /= Ntot;
  res->q_u = mu[0];
  res->q_v = mv[0];
  for (int d = 0; d < 3; ++d) {
    res->d_u[d] = mu[1 + d];
    res->d_v[d] = mv[1 + d];
    for (int e = 0; e < 3; ++e) {
      res->Q_u[d][e] = mu[4 + 3 * d + e];
      res->Q_v[d][e] = mv[4 + 3 * d + e];
    }
  }
  for (int u = 0; u < n; ++u)
    for (int d = 0; d < 3; ++d) res->d_n[d] += c->solute[u].charge * c->solute[u].x[d];
  double v1 = 0.0, v1l = 0.0;
  for (int u = 0; u < n; ++u) {
    const double q = c->solute[u].charge;
    v1 += q * val[u];
    double t = 0.0;
    for (int k = 0; k < 8; ++k) {
      const double wx = (k & 1) ? fr[3 * u] : 1 - fr[3 * u];
      const double wy = ((k >> 1) & 1) ? fr[3 * u + 1] : 1 - fr[3 * u + 1];
      const double wz = (k >> 2) ? fr[3 * u + 2] : 1 - fr[3 * u + 2];
      t += wx * wy * wz * val[n + 8 * u + k];
    }
    v1l += q * t;
    if (site_potential) site_potential[u] = val[u];
  }
  res->U_v_rho_N = v1;
  res->U_v_rho_N_trilinear = v1l;
  // Parseval: h^3 sum v_e rho_u = (h^3 / N) sum_k V conj(Ru) over the full spectrum
  res->U_v_rho_u = c->h3 * val[npts] / Ntot;
  double d3 = 0.0;
  for (double x : hd) d3 += x;
  res->rho_v_U_u = c->h3 * d3;
  res->seconds = ms * 1e-3;
  return RISM3D_OK;
}

// Device -> host copy of a large result into caller memory that is
// pageable (a NumPy array, a PETSc Vec): the driver's pageable path runs at
// a few GB/s there.  Here the copy is split into kLanes contiguous slices,
// each run by its own host thread on its own stream through two alternating
// pinned pieces: the DMA of piece i of a slice runs while its thread copies
// piece i-1 out, and the lanes run side by side, so the PCIe transfer and
// the host copy (402 MB: 7 ms and, on 8 threads, 5.5 ms on the B200 hosts)
// overlap instead of alternating.  The lane sets (kLanes streams and 2 x
// kLanes pieces of kPiece bytes: 64 MB pinned) come from a process-wide free
// list, one per concurrent caller, held until exit.  Copies below 32 MB take
// the plain cudaMemcpy.
constexpr size_t kPiece = size_t(4) << 20;
constexpr int kLanes = 8;
struct LaneSet {
  void *buf[kLanes][2] = {};
  cudaStream_t st[kLanes] = {};
  cudaEvent_t ev[kLanes][2] = {};
};
std::mutex g_stage_mu;
std::vector<LaneSet *> g_stage_free;

LaneSet *lane_set_new() {
  auto *ls = new LaneSet;
  try {
    for (int l = 0; l < kLanes; ++l) {
      for (int b = 0; b < 2; ++b) {
        CK(cudaHostAlloc(&ls->buf[l][b], kPiece, cudaHostAllocPortable));
        CK(cudaEventCreateWithFlags(&ls->ev[l][b], cudaEventDisableTiming));
      }
      CK(cudaStreamCreateWithFlags(&ls->st[l], cudaStreamNonBlocking));
    }
  } catch (...) {
    for (int l = 0; l < kLanes; ++l) {
      for (int b = 0; b < 2; ++b) {
        if (ls->buf[l][b]) cudaFreeHost(ls->buf[l][b]);
        if (ls->ev[l][b]) cudaEventDestroy(ls->ev[l][b]);
      }
      if (ls->st[l]) cudaStreamDestroy(ls->st[l]);
    }
    delete ls;
    throw;
  }
  return ls;
}

LaneSet *lane_set_take() {
  {
    std::lock_guard<std::mutex> lk(g_stage_mu);
    if (!g_stage_free.empty()) {
      LaneSet *ls = g_stage_free.back();
      g_stage_free.pop_back();
      return ls;
    }
  }
  return lane_set_new();
}

// Runs lane(l) for l < kLanes, lanes 1.. on their own threads.
template <typename F> void run_lanes(F &&lane) {
  std::vector<std::thread> th;
  for (int l = 1; l < kLanes; ++l) {
    try {
      th.emplace_back(lane, l);
    } catch (const std::system_error &) {  // no thread to be had: run the lane here
      lane(l);
    }
  }
  lane(0);
  for (auto &t : th) t.join();
}

// The set goes back only once none of its streams can still be moving data.
void lane_set_give(LaneSet *ls, bool failed) {
  bool clean = !failed;
  for (int l = 0; l < kLanes; ++l) clean = clean && cudaStreamSynchronize(ls->st[l]) == cudaSuccess;
  if (clean) {
    std::lock_guard<std::mutex> lk(g_stage_mu);
    g_stage_free.push_back(ls);
  }
  if (failed) {
    g_last_error = std::string("staged host copy failed: ") + cudaGetErrorString(cudaGetLastError());
    throw CudaFail{RISM3D_ERR_CUDA};
  }
}

// Host -> device copy of a large input from pageable caller memory: each
// lane copies a piece into pinned memory and moves it while it fills the
// other; complete (and ordered before later work on st) on return.
void h2d_large(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (bytes < (size_t(32) << 20)) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return;
  }
  LaneSet *ls = lane_set_take();
  cudaEvent_t ready = nullptr;  // dst (stream-ordered on st) exists
  CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  CK(cudaEventRecord(ready, st));
  std::atomic<int> failed{0};
  const size_t slice = ((bytes + kLanes - 1) / kLanes + kPiece - 1) / kPiece * kPiece;
  run_lanes([&](int l) {
    const size_t a = std::min(bytes, (size_t)l * slice), b = std::min(bytes, a + slice);
    if (a >= b) return;
    if (cudaStreamWaitEvent(ls->st[l], ready, 0) != cudaSuccess) { failed = 1; return; }
    size_t i = 0;
    for (size_t off = a; off < b; off += kPiece, ++i) {
      const size_t len = std::min(kPiece, b - off);
      // the DMA that last read this buffer (two pieces ago) has finished
      if (i >= 2 && cudaEventSynchronize(ls->ev[l][i & 1]) != cudaSuccess) { failed = 1; return; }
      std::memcpy(ls->buf[l][i & 1], static_cast<const char *>(src) + off, len);
      if (cudaMemcpyAsync(static_cast<char *>(dst) + off, ls->buf[l][i & 1], len, cudaMemcpyHostToDevice,
                          ls->st[l]) != cudaSuccess ||
          cudaEventRecord(ls->ev[l][i & 1], ls->st[l]) != cudaSuccess) {
        failed = 1;
        return;
      }
    }
  });
  cudaEventDestroy(ready);
  lane_set_give(ls, failed != 0);
}

void d2h_large(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (bytes < (size_t(32) << 20)) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return;
  }
  LaneSet *ls = lane_set_take();
  // the lanes' streams start once the source is complete on st
  cudaEvent_t ready = nullptr;
  CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  CK(cudaEventRecord(ready, st));
  std::atomic<int> failed{0};
  const size_t slice = ((bytes + kLanes - 1) / kLanes + kPiece - 1) / kPiece * kPiece;
  auto lane = [&](int l) {
    const size_t a = std::min(bytes, (size_t)l * slice), b = std::min(bytes, a + slice);
    if (a >= b) return;
    if (cudaStreamWaitEvent(ls->st[l], ready, 0) != cudaSuccess) { failed = 1; return; }
    size_t prev_off = 0, prev_len = 0;
    for (size_t off = a, i = 0;; off += kPiece, ++i) {
      const bool more = off < b;
      const size_t len = more ? std::min(kPiece, b - off) : 0;
      if (more) {
        if (cudaMemcpyAsync(ls->buf[l][i & 1], static_cast<const char *>(src) + off, len, cudaMemcpyDeviceToHost,
                            ls->st[l]) != cudaSuccess ||
            cudaEventRecord(ls->ev[l][i & 1], ls->st[l]) != cudaSuccess) {
          failed = 1;
          return;
        }
      }
      if (i > 0) {  // piece i-1 out of its buffer while piece i is in flight
        if (cudaEventSynchronize(ls->ev[l][(i - 1) & 1]) != cudaSuccess) { failed = 1; return; }
        std::memcpy(static_cast<char *>(dst) + prev_off, ls->buf[l][(i - 1) & 1], prev_len);
      }
      if (!more) break;
      prev_off = off;
      prev_len = len;
    }
  };
  run_lanes(lane);
  cudaEventDestroy(ready);
  lane_set_give(ls, failed != 0);
}

// Contexts of finished host-buffer solves, kept for the next
// rism3d_solute_solve with the same device, problem settings, solvent and
// chi: that call rebinds the solute (its short-range field and long-range
// term) instead of building the context again -- the grids, chi tables,
// coarse problem, transfer tables, Krylov buffers and the captured coarse
// solve are reused, as FFT plan caches reuse plans.  At most
// RISM3D_CTX_CACHE contexts (default 1, 0: off) are kept, least recently
// used first out; rism3d_cache_clear() frees them.  A context is taken out
// of the cache while a solve runs on it, so concurrent callers never share
// one.
struct CacheKey {
  int dev = -1;
  rism3d_problem pd{};
  std::vector<rism3d_site> solvent;
  std::vector<double> chi;  // [m][m][nrad]
};
struct CacheEntry {
  CacheKey key;
  rism3d_ctx *ctx;
};
std::mutex g_cache_mu;
std::vector<CacheEntry> g_cache;  // most recently used last

size_t cache_capacity() {
  static const size_t cap = [] {
    const char *e = std::getenv("RISM3D_CTX_CACHE");
    return e ? (size_t)std::max(0, std::atoi(e)) : size_t(1);
  }();
  return cap;
}

bool same_problem(const rism3d_problem &a, const rism3d_problem &b) {
  for (int i = 0; i < 3; ++i)
    if (a.N[i] != b.N[i] || a.L[i] != b.L[i]) return false;
  return a.beta == b.beta && a.rho == b.rho && a.rmax == b.rmax && a.nrad == b.nrad && a.closure == b.closure &&
         a.max_iter == b.max_iter && a.norm_tol == b.norm_tol && a.lambda == b.lambda && a.solver == b.solver &&
         a.renorm == b.renorm && a.precision == b.precision && a.verbosity == b.verbosity &&
         a.krylov_restart == b.krylov_restart && a.ew_forcing == b.ew_forcing && a.coarse_h == b.coarse_h &&
         a.coarse_steps == b.coarse_steps;
}

bool same_sites(const rism3d_site *a, const rism3d_site *b, int n) {
  for (int i = 0; i < n; ++i)
    if (a[i].x[0] != b[i].x[0] || a[i].x[1] != b[i].x[1] || a[i].x[2] != b[i].x[2] || a[i].sigma != b[i].sigma ||
        a[i].epsilon != b[i].epsilon || a[i].charge != b[i].charge)
      return false;
  return true;
}

rism3d_ctx *cache_take(const rism3d_problem *pd, int m, const rism3d_site *solvent, const double *chi) {
  if (cache_capacity() == 0) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  const size_t nchi = (size_t)m * m * (size_t)std::max(pd->nrad, 0);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  for (size_t i = g_cache.size(); i-- > 0;) {
    const CacheKey &k = g_cache[i].key;
    if (k.dev != dev || (int)k.solvent.size() != m || k.chi.size() != nchi || !same_problem(k.pd, *pd) ||
        !same_sites(k.solvent.data(), solvent, m) || std::memcmp(k.chi.data(), chi, sizeof(double) * nchi) != 0)
      continue;
    rism3d_ctx *c = g_cache[i].ctx;
    g_cache.erase(g_cache.begin() + (long)i);
    return c;
  }
  return nullptr;
}

void cache_put(rism3d_ctx *c, const rism3d_problem *pd, int m, const rism3d_site *solvent, const double *chi) {
  const size_t cap = cache_capacity();
  int dev = 0;
  if (cap == 0 || cudaGetDevice(&dev) != cudaSuccess) {
    delete c;
    return;
  }
  CacheEntry e{CacheKey{}, c};
  e.key.dev = dev;
  e.key.pd = *pd;
  e.key.solvent.assign(solvent, solvent + m);
  e.key.chi.assign(chi, chi + (size_t)m * m * (size_t)std::max(pd->nrad, 0));
  std::vector<rism3d_ctx *> drop;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache.push_back(std::move(e));
    while (g_cache.size() > cap) {
      drop.push_back(g_cache.front().ctx);
      g_cache.erase(g_cache.begin());
    }
  }
  for (auto *d : drop) delete d;
}

void cache_clear() {
  std::vector<CacheEntry> all;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    all.swap(g_cache);
  }
  for (auto &e : all) delete e.ctx;
}

// Writes one byte into every page of [p, p + bytes) from a few host threads:
// a caller's fresh result buffer (a NumPy array) takes its first-touch page
// faults here, while the device solves, instead of inside the copy-out.
struct PageToucher {
  std::vector<std::thread> th;
  PageToucher(void *p, size_t bytes) {
    if (!p || bytes < (size_t(64) << 20)) return;
    const long pg = 4096;
    const int nthr = 4;
    const size_t slice = (bytes / nthr + pg - 1) / pg * pg;
    for (int q = 0; q < nthr; ++q) {
      const size_t a = std::min(bytes, q * slice), b = std::min(bytes, (q + 1) * slice);
      if (a >= b) continue;
      try {
        th.emplace_back([=] {
          volatile char *c = static_cast<char *>(p);
          for (size_t o = a; o < b; o += pg) c[o] = 0;
        });
      } catch (const std::system_error &) {
        break;  // no thread: the copy-out takes the faults
      }
    }
  }
  void join() {
    for (auto &t : th) t.join();
    th.clear();
  }
  ~PageToucher() { join(); }
};

// One solve on a context from host buffers (rism3d_solute_solve).
int solve_on(rism3d_ctx *ctx, double *t_inout, double *g_out, rism3d_result *out) {
  const size_t bytes = sizeof(double) * ctx->nvec;
  double *T = dalloc<double>(ctx->nvec);
  double *g = g_out ? dalloc<double>(ctx->nvec) : nullptr;
  struct Free { double *a, *b; ~Free() { dfree(a); dfree(b); } } fr{T, g};
  if (t_inout) h2d_large(T, t_inout, bytes, ctx->stream);
  else CK(cudaMemsetAsync(T, 0, bytes, ctx->stream));
  PageToucher touch(g_out, bytes);  // g_out is written in full below; its old contents do not matter
  rism3d_result r{};
  int st = solve_impl(ctx, T, &r);
  observables_impl(ctx, T, g, &r);
  r.launches += 2;  // the observables' kernels
  r.status = st;
  touch.join();
  if (t_inout) d2h_large(t_inout, T, bytes, ctx->stream);
  if (g_out) d2h_large(g_out, g, bytes, ctx->stream);
  if (out) *out = r;
  return st;
}

template <typename F> int guard(F &&f) {
  try {
    return f();
  } catch (const CudaFail &e) {
    return e.code;
  } catch (const ArgFail &e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    g_last_error = "host allocation failed";
    return RISM3D_ERR_NOMEM;
  }
}

}  // namespace

namespace rism {
// Records the message that rism3d_last_error() returns on this thread (for
// the library's other translation units).
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace rism

// ================================================================== C ABI
extern "C" {

void rism3d_problem_defaults(rism3d_problem *pd, double L_half, int N) {
  std::memset(pd, 0, sizeof(*pd));
  for (int d = 0; d < 3; ++d) {
    pd->N[d] = N;
    pd->L[d] = 2 * L_half;
  }
  pd->beta = 1.6889;
  pd->rho = 0.033427745;
  pd->rmax = 2 * L_half / 2;
  pd->nrad = N;
  pd->closure = RISM3D_HNC;
  pd->max_iter = 1500;
  pd->norm_tol = 1.0e-7;
  pd->lambda = 0.02;
  pd->solver = RISM3D_NEWTON;
  pd->renorm = 1;
  pd->precision = RISM3D_FP64;
  pd->verbosity = 0;
  pd->krylov_restart = 30;
  pd->ew_forcing = 1;
  pd->coarse_h = 0.75;
  pd->coarse_steps = 16;
}

const char *rism3d_last_error(void) { return g_last_error.c_str(); }

int rism3d_ctx_create(const rism3d_problem *pd, int m, const rism3d_site *solvent, int n,
                      const rism3d_site *solute, const double *chi, rism3d_ctx **ctx) {
  if (ctx) *ctx = nullptr;
  return guard([&] { return create_impl(pd, m, solvent, n, solute, chi, nullptr, ctx); });
}

void rism3d_ctx_destroy(rism3d_ctx *ctx) { delete ctx; }

long long rism3d_ctx_size(const rism3d_ctx *ctx) { return ctx ? ctx->nvec : 0; }

int rism3d_iterate_t1(rism3d_ctx *ctx, const double *T, double *dT, double *resid) {
  if (!ctx || !T || !dT) return RISM3D_ERR_ARG;
  return guard([&] {
    double r[2];
    eval_F<double>(ctx, T, dT, r);
    if (resid) resid[0] = r[0], resid[1] = r[1];
    return RISM3D_OK;
  });
}

int rism3d_jacobian_t1(rism3d_ctx *ctx, const double *T, const double *dT, double *JdT) {
  if (!ctx || !T || !dT || !JdT) return RISM3D_ERR_ARG;
  if (ctx->pd.closure == RISM3D_PY) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] {
    double *d = slopebuf<double>(ctx);
    if (ctx->pure) eval_F<double>(ctx, T, JdT, nullptr);  // C(k) at T for the OZ differential
    closure_slope<double, double>(ctx, T, d);
    eval_J<double>(ctx, d, dT, 1.0, JdT, nullptr);
    CK(cudaStreamSynchronize(ctx->stream));
    return RISM3D_OK;
  });
}

int rism3d_iterate_t1_f32(rism3d_ctx *ctx, const float *T, float *dT, double *resid) {
  if (!ctx || !T || !dT) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] {
    double r[2];
    eval_F<float>(ctx, T, dT, r);
    if (resid) resid[0] = r[0], resid[1] = r[1];
    return RISM3D_OK;
  });
}

int rism3d_jacobian_t1_f32(rism3d_ctx *ctx, const float *T, const float *dT, float *JdT) {
  if (ctx && ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  if (!ctx || !T || !dT || !JdT) return RISM3D_ERR_ARG;
  if (ctx->pd.closure == RISM3D_PY) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] {
    float *d = slopebuf<float>(ctx);
    closure_slope<float, float>(ctx, T, d);
    eval_J<float>(ctx, d, dT, 1.0, JdT, nullptr);
    CK(cudaStreamSynchronize(ctx->stream));
    return RISM3D_OK;
  });
}

int rism3d_solve(rism3d_ctx *ctx, double *T, rism3d_result *out) {
  if (!ctx || !T) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] { return solve_impl(ctx, T, out); });
}

int rism3d_observables(rism3d_ctx *ctx, const double *T, double *g, rism3d_result *out) {
  if (!ctx || !T) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] { return observables_impl(ctx, T, g, out); });
}

int rism3d_get_field(rism3d_ctx *ctx, int which, double *dst) {
  if (!ctx || !dst) return RISM3D_ERR_ARG;
  return guard([&] {
    if (which == 0) {
      CK(cudaMemcpy(dst, ctx->v64, sizeof(double) * ctx->nvec, cudaMemcpyDeviceToDevice));
    } else if (which == 1) {
      const rism3d_problem &pd = ctx->pd;
      const unsigned nb = (unsigned)((ctx->g.Nr + 255) / 256);
      k_coulomb_long<<<nb, 256, 0, ctx->stream>>>(ctx->g, pd.L[0] / pd.N[0], pd.L[1] / pd.N[1], pd.L[2] / pd.N[2],
                                                  pd.L[0], pd.L[1], pd.L[2], ctx->n, ctx->d_solute, dst);
      CKL();
      CK(cudaStreamSynchronize(ctx->stream));
    } else {
      return (int)RISM3D_ERR_ARG;
    }
    return (int)RISM3D_OK;
  });
}

int rism3d_solute_solve(const rism3d_problem *pd, int m, const rism3d_site *solvent, int n,
                        const rism3d_site *solute, const double *chi, double *t_inout, double *g_out,
                        rism3d_result *out) {
  int rc = RISM3D_OK;
  rism3d_ctx *ctx = nullptr;
  if (pd && solvent && chi && m >= 1 && m <= kMaxSites && n >= 0 && (solute || n == 0)) {
    ctx = cache_take(pd, m, solvent, chi);
    if (ctx) {
      rc = guard([&] {
        bind_solute(ctx, n, solute);
        return (int)RISM3D_OK;
      });
      if (rc != RISM3D_OK) {
        delete ctx;
        ctx = nullptr;
      }
    }
  }
  if (!ctx) {
    rc = rism3d_ctx_create(pd, m, solvent, n, solute, chi, &ctx);
    if (rc != RISM3D_OK) {
      if (out) { std::memset(out, 0, sizeof(*out)); out->status = rc; }
      return rc;
    }
  }
  rc = guard([&] { return solve_on(ctx, t_inout, g_out, out); });
  if (rc == RISM3D_OK || rc == RISM3D_ERR_NOT_CONVERGED || rc == RISM3D_ERR_NAN)
    cache_put(ctx, pd, m, solvent, chi);
  else
    rism3d_ctx_destroy(ctx);
  if (out && rc < 0 && out->status == 0) out->status = rc;
  return rc;
}

void rism3d_cache_clear(void) { cache_clear(); }

int rism3d_tile_shapes(rism3d_ctx *ctx, int *out) {
  if (!ctx || !out) return RISM3D_ERR_ARG;
  for (int pr = 0; pr < 2; ++pr) {
    out[3 * pr] = ctx->tiles[pr].RX;
    out[3 * pr + 1] = ctx->tiles[pr].BY;
    out[3 * pr + 2] = ctx->tiles[pr].BZ;
    out[6 + pr] = ctx->stat[pr] ? 1 : 0;
    out[8 + pr] = ctx->zb[pr] * (ctx->zpers[pr] ? -1 : 1);  // negative: persistent CTAs
  }
  return RISM3D_OK;
}

int rism3d_info(rism3d_ctx *ctx, const double *T, rism3d_info_result *out, double *site_potential) {
  if (!ctx || !T || !out) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] { return info_impl(ctx, T, out, site_potential); });
}

int rism3d_moments(rism3d_ctx *ctx, const double *g, int fields, double *out) {
  if (!ctx || !g || !out || fields < 1) return RISM3D_ERR_ARG;
  return guard([&] {
    moments_of(ctx, g, fields, 1.0, -1.0, out);
    return RISM3D_OK;
  });
}

int rism3d_ctx_create_chi3(const rism3d_problem *pd, int m, const rism3d_site *solvent, int n,
                           const rism3d_site *solute, const double *chi3, rism3d_ctx **ctx) {
  if (ctx) *ctx = nullptr;
  if (!chi3) return RISM3D_ERR_ARG;
  return guard([&] { return create_impl(pd, m, solvent, n, solute, nullptr, chi3, ctx); });
}

int rism3d_solute_solve_chi3(const rism3d_problem *pd, int m, const rism3d_site *solvent, int n,
                             const rism3d_site *solute, const double *chi3, double *t_inout, double *g_out,
                             rism3d_result *out) {
  rism3d_ctx *ctx = nullptr;
  int rc = rism3d_ctx_create_chi3(pd, m, solvent, n, solute, chi3, &ctx);
  if (rc != RISM3D_OK) {
    if (out) { std::memset(out, 0, sizeof(*out)); out->status = rc; }
    return rc;
  }
  rc = guard([&] { return solve_on(ctx, t_inout, g_out, out); });
  rism3d_ctx_destroy(ctx);
  if (out && rc < 0 && out->status == 0) out->status = rc;
  return rc;
}

int rism3d_solvent_ctx_create(const rism3d_problem *pd, int m, const rism3d_site *solvent, rism3d_ctx **ctx) {
  if (ctx) *ctx = nullptr;
  return guard([&] { return solvent_create_impl(pd, m, solvent, ctx); });
}

int rism3d_solvent_solve(const rism3d_problem *pd, int m, const rism3d_site *solvent, const double *t_in,
                         double *t_out, double *chi_out, double *g_out, rism3d_solvent_result *out) {
  rism3d_solvent_result res{};
  rism3d_ctx *ctx = nullptr;
  int rc = rism3d_solvent_ctx_create(pd, m, solvent, &ctx);
  if (rc == RISM3D_OK) {
    rc = guard([&] {
      const size_t bytes = sizeof(double) * ctx->nvec;
      double *T = dalloc<double>(ctx->nvec);
      struct Free { double *a; ~Free() { dfree(a); } } fr{T};
      if (t_in) CK(cudaMemcpy(T, t_in, bytes, cudaMemcpyHostToDevice));
      else solvent_guess(ctx, T);
      const int st = solvent_solve_impl(ctx, T, chi_out, g_out, &res);
      if (t_out) CK(cudaMemcpy(t_out, T, bytes, cudaMemcpyDeviceToHost));
      return st;
    });
    rism3d_ctx_destroy(ctx);
  }
  if (res.status == 0) res.status = rc;
  if (out) *out = res;
  return rc;
}

int rism3d_solve_batch(int m, const rism3d_site *solvent, int njobs, rism3d_job *jobs, int workers) {
  if (njobs < 0 || (njobs > 0 && !jobs) || !solvent || m < 1) return RISM3D_ERR_ARG;
  if (njobs == 0) return RISM3D_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RISM3D_ERR_CUDA;
  const int nw = std::max(1, std::min(workers > 0 ? workers : 8, njobs));
  // largest grids first, so that the last jobs to start are short ones
  std::vector<int> order(njobs);
  std::iota(order.begin(), order.end(), 0);
  auto cost = [&](int i) {
    const rism3d_problem &p = jobs[i].pd;
    return (double)p.N[0] * p.N[1] * p.N[2];
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  std::atomic<int> next{0};
  auto work = [&] {
    // each worker issues on its own per-thread default stream
    if (cudaSetDevice(dev) != cudaSuccess) return;
    tl_concurrent_solves = nw > 1;
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= njobs) break;
      rism3d_job &j = jobs[order[i]];
      rism3d_solute_solve(&j.pd, m, solvent, j.n, j.solute, j.chi, j.t_inout, j.g_out, &j.result);
    }
    cudaStreamSynchronize(cudaStreamPerThread);
  };
  std::vector<std::thread> pool;
  pool.reserve(nw);
  for (int w = 0; w < nw; ++w) pool.emplace_back(work);
  for (auto &t : pool) t.join();
  int rc = RISM3D_OK;
  for (int i = 0; i < njobs && rc == RISM3D_OK; ++i) rc = jobs[i].result.status;
  return rc;
}

int rism3d_ctx_set_solute(rism3d_ctx *ctx, int n, const rism3d_site *solute) {
  if (!ctx || n < 0 || (n > 0 && !solute)) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] {
    bind_solute(ctx, n, solute);
    return (int)RISM3D_OK;
  });
}

int rism3d_jacobian_transpose_t1(rism3d_ctx *ctx, const double *T, const double *dT, double *JT) {
  if (!ctx || !T || !dT || !JT) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] { return jacobian_transpose_impl(ctx, T, dT, JT); });
}

int rism3d_gradient(rism3d_ctx *ctx, const double *T, rism3d_grad *grad) {
  if (!ctx || !T || !grad) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] {
    int rc = gradient_impl(ctx, T, grad);
    if (rc == RISM3D_OK && grad->dx_reference) rc = reference_gradient_impl(ctx, T, grad->dx_reference);
    return rc;
  });
}

int rism3d_free_energy_gradient(rism3d_ctx *ctx, const double *T, double *de) {
  if (!ctx || !T || !de) return RISM3D_ERR_ARG;
  return guard([&] { return reference_gradient_impl(ctx, T, de); });
}

int rism3d_response(rism3d_ctx *ctx, const double *T, rism3d_grad *grad) {
  if (!ctx || !T || !grad) return RISM3D_ERR_ARG;
  if (ctx->pure) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] { return response_impl(ctx, T, grad); });
}

int rism3d_solute_grad(const rism3d_problem *pd, int m, const rism3d_site *solvent, int n,
                       const rism3d_site *solute, const double *chi, double *t_inout, rism3d_result *out,
                       rism3d_grad *grad) {
  if (!grad) return RISM3D_ERR_ARG;
  if (pd && !pd->renorm) {
    g_last_error = "the gradient is implemented for the renormalised form only";
    return RISM3D_ERR_UNSUPPORTED;
  }
  rism3d_ctx *ctx = nullptr;
  int rc = rism3d_ctx_create(pd, m, solvent, n, solute, chi, &ctx);
  if (rc != RISM3D_OK) {
    if (out) { std::memset(out, 0, sizeof(*out)); out->status = rc; }
    return rc;
  }
  rc = guard([&] {
    const size_t bytes = sizeof(double) * ctx->nvec;
    double *T = dalloc<double>(ctx->nvec);
    struct Free { double *a; ~Free() { dfree(a); } } fr{T};
    if (t_inout) CK(cudaMemcpy(T, t_inout, bytes, cudaMemcpyHostToDevice));
    else CK(cudaMemset(T, 0, bytes));
    rism3d_result r{};
    int st = solve_impl(ctx, T, &r);
    observables_impl(ctx, T, nullptr, &r);
    r.status = st;
    if (st == RISM3D_OK) st = gradient_impl(ctx, T, grad);
    if (st == RISM3D_OK && grad->dx_reference) st = reference_gradient_impl(ctx, T, grad->dx_reference);
    if (t_inout) CK(cudaMemcpy(t_inout, T, bytes, cudaMemcpyDeviceToHost));
    if (out) *out = r;
    return st;
  });
  rism3d_ctx_destroy(ctx);
  if (out && rc < 0 && out->status == 0) out->status = rc;
  return rc;
}

int rism3d_precondition(rism3d_ctx *ctx, const double *T, const double *v, double *z) {
  if (!ctx || !T || !v || !z) return RISM3D_ERR_ARG;
  if (!ctx->coarse) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] {
    double *d = slopebuf<double>(ctx);
    closure_slope<double, double>(ctx, T, d);
    tg_prepare<double>(ctx, d);
    tg_apply<double>(ctx, v, 1.0, z);
    CK(cudaStreamSynchronize(ctx->stream));
    return (int)RISM3D_OK;
  });
}

int rism3d_precondition_f32(rism3d_ctx *ctx, const float *T, const float *v, float *z) {
  if (!ctx || !T || !v || !z) return RISM3D_ERR_ARG;
  if (!ctx->coarse) return RISM3D_ERR_UNSUPPORTED;
  return guard([&] {
    float *d = slopebuf<float>(ctx);
    closure_slope<float, float>(ctx, T, d);
    tg_prepare<float>(ctx, d);
    tg_apply<float>(ctx, v, 1.0, z);
    CK(cudaStreamSynchronize(ctx->stream));
    return (int)RISM3D_OK;
  });
}

int rism3d_coarse_grid(rism3d_ctx *ctx, int *n) {
  if (!ctx || !n) return RISM3D_ERR_ARG;
  for (int a = 0; a < 3; ++a) n[a] = ctx->coarse ? ctx->Nc[a] : 0;
  return RISM3D_OK;
}

int rism3d_coarse_driver(rism3d_ctx *ctx) {
  if (!ctx) return RISM3D_ERR_ARG;
  return ctx->coarse_driver;
}

// ---- profiling hooks (per-pass CUDA-event timing, off by default) -------
int rism3d_profile(rism3d_ctx *ctx, int on, double *ms_out, long long *launches_out) {
  if (!ctx) return RISM3D_ERR_ARG;
  return guard([&] {
    if (ms_out)
      for (int i = 0; i < 12; ++i) ms_out[i] = ctx->timer.ms[i];
    if (launches_out)
      for (int i = 0; i < 12; ++i) launches_out[i] = ctx->timer.launches[i];
    if (on && !ctx->timer.on) {
      CK(cudaEventCreate(&ctx->timer.a));
      CK(cudaEventCreate(&ctx->timer.b));
      ctx->timer.on = true;
    } else if (!on && ctx->timer.on) {
      cudaEventDestroy(ctx->timer.a);
      cudaEventDestroy(ctx->timer.b);
      ctx->timer.on = false;
    }
    for (int i = 0; i < 12; ++i) ctx->timer.ms[i] = 0, ctx->timer.launches[i] = 0;
    return (int)RISM3D_OK;
  });
}

}  // extern "C"
