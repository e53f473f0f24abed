// kernels_static.cuh -- shape-specialised FFT passes of the 3D-RISM residual
// (the same five passes as kernels.cuh, for compile-time transform lengths).
//
//   k_xfwd_s  closure (or its linearisation) + r2c along x: RX contiguous rows
//             per CTA, vector loads, padded shared-memory rows;
//   k_y_s     one [N1][B] column tile per CTA, loaded and stored by TMA;
//   k_z_s     the m [N2][B] tiles of one (ky, kx-block), TMA in and out, with
//             the OZ contraction between the forward and inverse transforms;
//   k_xinv_s  c2r along x with "- t" and the residual norms.
//
// B columns of a y/z tile are 128 bytes (16 float2 or 8 double2): one TMA box
// row per transform index, so every HBM access is a whole 128-byte line.
#pragma once
#include "fft_static.cuh"
#include "kernels.cuh"

namespace rism {

constexpr uint32_t kMbarPolls = 1u << 26;  // bounded mbarrier wait (seconds)

template <typename T> struct VecW;  // complex values per vector load in the x passes
template <> struct VecW<float> { static constexpr int n = 2; using vec = float4; };
template <> struct VecW<double> { static constexpr int n = 1; using vec = double2; };

// x forward (see k_xfwd): MODE_F c = closure(p B, A); MODE_J c = B (p A).
template <typename T, int MODE, int M, int RX>
__global__ void __launch_bounds__(256) k_xfwd_s(Geo g, const T *__restrict__ A, const T *__restrict__ Bv, T p,
                                               int closure, typename Cx<T>::type *__restrict__ W,
                                               const typename Cx<T>::type *__restrict__ post,
                                               const typename Cx<T>::type *__restrict__ twg) {
  using V = typename Cx<T>::type;
  using Lay = LayRow<M, SplitRow<M>::R2>;
  constexpr int VW = VecW<T>::n;
  using VEC = typename VecW<T>::vec;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + M;
  const int tid = threadIdx.x;
  const int rows_total = g.N1 * g.N2;
  const int row0 = blockIdx.x * RX;
  const int site = blockIdx.y;
  for (int q = tid; q < M; q += 256) tw[q] = twg[q];
  const long long sbase = (long long)site * g.Nr;
  constexpr int PER_ROW = M / VW;
  constexpr int CNT = (RX * PER_ROW + 255) / 256;
  // all loads of the thread in flight before any use
  VEC ra[CNT], rb[CNT];
#pragma unroll
  for (int it = 0; it < CNT; ++it) {
    const int e = tid + it * 256;
    const int row = e / PER_ROW, jj = (e % PER_ROW) * VW;
    if (e < RX * PER_ROW && row0 + row < rows_total) {
      const long long off = sbase + (long long)(row0 + row) * g.N0 + 2 * jj;
      ra[it] = *reinterpret_cast<const VEC *>(A + off);
      rb[it] = *reinterpret_cast<const VEC *>(Bv + off);
    }
  }
#pragma unroll
  for (int it = 0; it < CNT; ++it) {
    const int e = tid + it * 256;
    if (e >= RX * PER_ROW) break;
    const int row = e / PER_ROW, jj = (e % PER_ROW) * VW;
    const int grow = row0 + row;
    V z[VW];
#pragma unroll
    for (int v = 0; v < VW; ++v) z[v].x = z[v].y = T(0);
    if (grow < rows_total) {
      const T *ar = reinterpret_cast<const T *>(&ra[it]);
      const T *br = reinterpret_cast<const T *>(&rb[it]);
#pragma unroll
      for (int v = 0; v < VW; ++v) {
        if (MODE == MODE_F) {
          z[v].x = closure_c<T>(closure, p * br[2 * v], ar[2 * v]);
          z[v].y = closure_c<T>(closure, p * br[2 * v + 1], ar[2 * v + 1]);
        } else {
          z[v].x = br[2 * v] * (ar[2 * v] * p);
          z[v].y = br[2 * v + 1] * (ar[2 * v + 1] * p);
        }
      }
    }
#pragma unroll
    for (int v = 0; v < VW; ++v) buf[Lay::at(jj + v, row)] = z[v];
  }
  __syncthreads();
  fft2<M, RX, 256, false, false, Lay, SplitRow<M>>(buf, tw);
  constexpr int H = M / 2 + 1;
  const long long wbase = (long long)site * g.Nc;
  for (int e = tid; e < RX * H; e += 256) {
    const int row = e / H, k = e % H;
    const int grow = row0 + row;
    if (grow >= rows_total) continue;
    const V zk = buf[Lay::at(k, row)];
    const V zm = buf[Lay::at(k == 0 ? 0 : M - k, row)];
    V E, O;
    E.x = (zk.x + zm.x) * T(0.5);
    E.y = (zk.y - zm.y) * T(0.5);
    O.x = (zk.y + zm.y) * T(0.5);
    O.y = -(zk.x - zm.x) * T(0.5);
    const V wO = cmul(post[k], O);
    V *row_out = W + wbase + (long long)grow * g.Nhp;
    row_out[k] = cadd(E, wO);
    if (M - k != k) row_out[M - k] = cconj(csub(E, wO));
  }
}

// x inverse (see k_xinv): out = scale x - sub In, residual norms.
template <typename T, int M, int RX>
__global__ void __launch_bounds__(256) k_xinv_s(Geo g, const typename Cx<T>::type *__restrict__ W,
                                               const T *__restrict__ In, T *__restrict__ Out, T scale, T sub,
                                               const typename Cx<T>::type *__restrict__ post,
                                               const typename Cx<T>::type *__restrict__ twg,
                                               NormPartial *__restrict__ part) {
  using V = typename Cx<T>::type;
  using Lay = LayRow<M, SplitRow<M>::R2>;
  constexpr int VW = VecW<T>::n;
  using VEC = typename VecW<T>::vec;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + M;
  const int tid = threadIdx.x;
  const int rows_total = g.N1 * g.N2;
  const int row0 = blockIdx.x * RX;
  const int site = blockIdx.y;
  for (int q = tid; q < M; q += 256) tw[q] = twg[q];
  constexpr int H = M / 2 + 1;
  const long long wbase = (long long)site * g.Nc;
  const long long sbase = (long long)site * g.Nr;
  constexpr int PER_ROW = M / VW;
  constexpr int CNT = (RX * PER_ROW + 255) / 256;
  // the subtracted input is fetched first; its latency hides behind the
  // transform
  VEC rin[CNT];
#pragma unroll
  for (int it = 0; it < CNT; ++it) {
    const int e = tid + it * 256;
    const int row = e / PER_ROW, jj = (e % PER_ROW) * VW;
    if (e < RX * PER_ROW && row0 + row < rows_total)
      rin[it] = *reinterpret_cast<const VEC *>(In + sbase + (long long)(row0 + row) * g.N0 + 2 * jj);
  }
  // packed c2r input of element e = (row, k <= M/2) from X_k and X_{M-k}
  auto pack = [&](int e, V xk, V xm) {
    const int row = e / H, k = e % H;
    V zk, zm;
    zk.x = zk.y = zm.x = zm.y = T(0);
    if (row0 + row < rows_total) {
      if (k == 0) { xk.y = T(0); xm.y = T(0); }  // c2r reads only Re X_0, Re X_{N0/2}
      V Aa, D;
      Aa.x = xk.x + xm.x; Aa.y = xk.y - xm.y;
      D.x = xk.x - xm.x;  D.y = xk.y + xm.y;
      const V Pp = cmul(D, cconj(post[k]));
      zk.x = Aa.x - Pp.y; zk.y = Aa.y + Pp.x;
      zm.x = Aa.x + Pp.y; zm.y = -(Aa.y - Pp.x);
    }
    buf[Lay::at(k, row)] = zk;
    if (k != 0 && M - k != k) buf[Lay::at(M - k, row)] = zm;
  };
  auto ld = [&](int e, V &xk, V &xm) {
    const int row = e / H, k = e % H;
    if (row0 + row < rows_total) {
      const V *row_in = W + wbase + (long long)(row0 + row) * g.Nhp;
      xk = row_in[k];
      xm = row_in[M - k];
    } else {
      xk.x = xk.y = xm.x = xm.y = T(0);
    }
  };
  constexpr int CW = (RX * H + 255) / 256;
  if constexpr (CW <= 6) {
    // every (X_k, X_{M-k}) pair of this thread is loaded before the first is
    // used: one memory latency per CTA instead of one per pair of iterations
    // (longer rows keep the loop below: the registers would cost occupancy)
    V xkv[CW], xmv[CW];
#pragma unroll
    for (int it = 0; it < CW; ++it) {
      const int e = tid + it * 256;
      if (e < RX * H) ld(e, xkv[it], xmv[it]);
    }
#pragma unroll
    for (int it = 0; it < CW; ++it) {
      const int e = tid + it * 256;
      if (e < RX * H) pack(e, xkv[it], xmv[it]);
    }
  } else {
#pragma unroll 2
    for (int e = tid; e < RX * H; e += 256) {
      const int row = e / H, k = e % H;
      const int grow = row0 + row;
      V zk, zm;
      zk.x = zk.y = zm.x = zm.y = T(0);
      if (grow < rows_total) {
        const V *row_in = W + wbase + (long long)grow * g.Nhp;
        V xk = row_in[k];
        V xm = row_in[M - k];
        if (k == 0) { xk.y = T(0); xm.y = T(0); }
        V Aa, D;
        Aa.x = xk.x + xm.x; Aa.y = xk.y - xm.y;
        D.x = xk.x - xm.x;  D.y = xk.y + xm.y;
        const V Pp = cmul(D, cconj(post[k]));
        zk.x = Aa.x - Pp.y; zk.y = Aa.y + Pp.x;
        zm.x = Aa.x + Pp.y; zm.y = -(Aa.y - Pp.x);
      }
      buf[Lay::at(k, row)] = zk;
      if (k != 0 && M - k != k) buf[Lay::at(M - k, row)] = zm;
    }
  }
  __syncthreads();
  fft2<M, RX, 256, true, false, Lay, SplitRow<M>>(buf, tw);
  double amax = 0.0, sum2 = 0.0;
#pragma unroll
  for (int it = 0; it < CNT; ++it) {
    const int e = tid + it * 256;
    if (e >= RX * PER_ROW) break;
    const int row = e / PER_ROW, jj = (e % PER_ROW) * VW;
    const int grow = row0 + row;
    if (grow >= rows_total) continue;
    const long long off = sbase + (long long)grow * g.N0 + 2 * jj;
    const T *ir = reinterpret_cast<const T *>(&rin[it]);
    VEC o;
    T *orr = reinterpret_cast<T *>(&o);
#pragma unroll
    for (int v = 0; v < VW; ++v) {
      const V z = buf[Lay::at(jj + v, row)];
      orr[2 * v] = z.x * scale - sub * ir[2 * v];
      orr[2 * v + 1] = z.y * scale - sub * ir[2 * v + 1];
    }
    *reinterpret_cast<VEC *>(Out + off) = o;
#pragma unroll
    for (int v = 0; v < 2 * VW; ++v) {
      const double ov = (double)orr[v];
      amax = fmax(amax, fabs(ov));
      sum2 += ov * ov;
    }
  }
  block_norms(amax, sum2, part + (blockIdx.y * gridDim.x + blockIdx.x));
}

// A TMA box spans at most 256 elements per dimension: tiles along a 512-point
// axis move as two boxes of kTmaRows rows.
constexpr int kTmaRows = 256;

// y pass: one [N][B] tile (kx0 .. kx0+B-1 at fixed z, site) by TMA.
// tm: W as {2 Nhp, N1, m N2} scalars, box {2B, N1, 1}.
template <typename T, bool INV, int N, int B>
__global__ void __launch_bounds__(Split<N>::R1 * B) k_y_s(Geo g, const __grid_constant__ CUtensorMap tm,
                                                         const typename Cx<T>::type *__restrict__ twg,
                                                         int *__restrict__ err) {
  using V = typename Cx<T>::type;
  constexpr int NTHR = Split<N>::R1 * B;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *buf = reinterpret_cast<V *>(smem_raw);
  V *tw = buf + N * B;
  uint64_t *bar = reinterpret_cast<uint64_t *>(tw + N);
  const int tid = threadIdx.x;
  const int kx0 = blockIdx.x * B, z = blockIdx.y, site = blockIdx.z;
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(bar, (uint32_t)(N * B * sizeof(V)));
#pragma unroll
    for (int c = 0; c < N; c += kTmaRows) tma_load_3d(buf + c * B, &tm, bar, 2 * kx0, c, site * g.N2 + z);
  }
  for (int q = tid; q < N; q += NTHR) tw[q] = twg[q];
  if (!cta_wait_tile(bar, 0, kMbarPolls, err, 1)) return;
  fft2<N, B, NTHR, INV, true, LayCol<N, B>>(buf, tw);
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int c = 0; c < N; c += kTmaRows) tma_store_3d(&tm, buf + c * B, 2 * kx0, c, site * g.N2 + z);
    tma_commit();
    tma_wait_read0();
  }
}

// Elements whose chi table entries a thread has in flight during the z
// contraction: 4 in the FP32 Jacobian pass, 2 where the residual's
// long-range terms or FP64 values take the registers (the FP32 passes stay
// within 128 registers, i.e. the 4 CTAs per SM that shared memory allows).
template <typename T, int MODE> __host__ __device__ constexpr int zpf_default() {
  return sizeof(T) == 4 && MODE == MODE_J ? 4 : 2;
}

// One z tile in shared memory: forward transform along z of the m [N][B]
// site columns, the OZ contraction with the radial chi-1 tables (+ the
// long-range terms in MODE_F), inverse transform; ends after a barrier.
// Run by the NTHR = R1 B threads tid of a group (act false: barriers only);
// JOINT: the MS site tiles (all allocated) transform as one MS B-column
// tile by R1 B MS threads.
//
// The contraction is software-pipelined: the table entries of an element
// depend only on where it sits on the k grid, so a thread keeps those of its
// next ZPF elements (and, in MODE_F, their long-range values) in flight
// while it contracts the current one, and issues the first ZPF before the
// forward transforms, under whose latency they arrive.  Same arithmetic in
// the same order as contracting element by element.
template <typename T, int MODE, int N, int B, int MS, bool JOINT = false, int ZPF = zpf_default<T, MODE>(),
          class S = Split<N>>
__device__ __forceinline__ void z_tile_g(const Geo &g, typename Cx<T>::type *buf, const typename Cx<T>::type *tw,
                                         const ZParams<T> &zp, int kx0, int y, int tid, bool act) {
  using V = typename Cx<T>::type;
  using P2 = typename Vec2<T>::type;
  constexpr int NTHR = S::R1 * B * (JOINT ? MS : 1);
  constexpr int NP = MS * (MS + 1) / 2;
  constexpr int NIT = (N * B + NTHR - 1) / NTHR;
  constexpr int D = NIT < ZPF ? NIT : ZPF;
  const int m = g.m;
  const int np = m * (m + 1) / 2;
  const int bw = min(B, g.Nh - kx0);
  const bool full = MODE == MODE_F && zp.L != nullptr;
  const int ky = kfreq(y, g.N1);
  const double k1 = ky * g.dk1;
  const long long zstride = (long long)g.N1 * g.Nhp;
  const long long col = (long long)y * g.Nhp + kx0;
  P2 tq[D][NP];   // chi - 1 (value, slope) of each pair
  P2 sq[D][MS];   // beta/eps0 s_i (value, slope), MODE_F
  V lq[D];        // long-range value, MODE_F
  T fq[D];        // interpolation fraction
  auto fetch = [&](int it, int slot) {
    const int e = tid + it * NTHR;
    if (!act || e >= N * B) return;
    const int z = e / B, b = e % B;
    const int kx = kx0 + b;
    const int kz = kfreq(z, N);
    const double k0 = kx * g.dk0, k2 = kz * g.dk2;
    const double kk = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)), __dmul_rn(k2, k2)));
    const double ix = kk / zp.dkr - 0.5;
    int i = (int)(ix + 0.5);
    i = min(max(i, 0), zp.nrad - 1);
    fq[slot] = T(ix - i);
#pragma unroll
    for (int q = 0; q < NP; ++q)
      if (q < np) tq[slot][q] = __ldg(&zp.chi[(long long)q * zp.nrad + i]);
    lq[slot].x = T(0); lq[slot].y = T(0);
    if (full) {
      if (zp.stab != nullptr) {
#pragma unroll
        for (int ii = 0; ii < MS; ++ii)
          if (ii < m) sq[slot][ii] = __ldg(&zp.stab[(long long)ii * zp.nrad + i]);
      }
      if (b < bw) lq[slot] = __ldg(&zp.L[z * zstride + col + b]);
    }
  };
#pragma unroll
  for (int s = 0; s < D; ++s) fetch(s, s);
  if (JOINT) fft2g<N, MS * B, NTHR, false, true, LayCol<N, B>, S>(buf, tw, tid, act);
  else
    for (int s = 0; s < m; ++s) fft2g<N, B, NTHR, false, true, LayCol<N, B>, S>(buf + s * N * B, tw, tid, act);
#pragma unroll
  for (int it = 0; it < NIT; ++it) {
    const int slot = it % D;
    const int e = tid + it * NTHR;
    if (act && e < N * B) {
      const int b = e % B;
      const bool valid = b < bw;
      const T fr = fq[slot];
      const V Lk = lq[slot];
      V c[MS];
#pragma unroll
      for (int j = 0; j < MS; ++j)
        if (j < m) c[j] = buf[j * N * B + e];
      if (full) {
#pragma unroll
        for (int j = 0; j < MS; ++j)
          if (j < m) { c[j].x -= zp.a[j] * Lk.x; c[j].y -= zp.a[j] * Lk.y; }
      }
      T xv[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q)
        if (q < np) xv[q] = tq[slot][q].x + tq[slot][q].y * fr;
#pragma unroll
      for (int ii = 0; ii < MS; ++ii) {
        if (ii < m) {
          V t;
          t.x = T(0); t.y = T(0);
#pragma unroll
          for (int j = 0; j < MS; ++j) {
            if (j < m) {
              const T x = xv[ii >= j ? ii * (ii + 1) / 2 + j : j * (j + 1) / 2 + ii];
              t.x += x * c[j].x;
              t.y += x * c[j].y;
            }
          }
          if (full) {
            T bb = zp.bconst[ii];
            if (zp.stab != nullptr) bb += sq[slot][ii].x + sq[slot][ii].y * fr;
            t.x -= bb * Lk.x;
            t.y -= bb * Lk.y;
          }
          if (valid) buf[ii * N * B + e] = t;
        }
      }
    }
    if (it + D < NIT) fetch(it + D, slot);
  }
  __syncthreads();
  if (JOINT) fft2g<N, MS * B, NTHR, true, true, LayCol<N, B>, S>(buf, tw, tid, act);
  else
    for (int s = 0; s < m; ++s) fft2g<N, B, NTHR, true, true, LayCol<N, B>, S>(buf + s * N * B, tw, tid, act);
}
template <typename T, int MODE, int N, int B, int MS>
__device__ __forceinline__ void z_tile(const Geo &g, typename Cx<T>::type *buf, const typename Cx<T>::type *tw,
                                       const ZParams<T> &zp, int kx0, int y) {
  z_tile_g<T, MODE, N, B, MS>(g, buf, tw, zp, kx0, y, (int)threadIdx.x, true);
}

// z pass: the m [N][B] tiles of one (ky, kx-block) by TMA, forward transform,
// OZ contraction (+ long-range terms in MODE_F), inverse transform, TMA out.
// tm: W as {2 Nhp, N1, m N2} scalars, box {2B, 1, N2}.
template <typename T, int MODE, int N, int B, int MS>
__global__ void __launch_bounds__(Split<N>::R1 * B, sizeof(T) == 4 ? 4 : 1) k_z_s(Geo g,
                                                                                  const __grid_constant__ CUtensorMap tm,
                                                         const typename Cx<T>::type *__restrict__ twg,
                                                         ZParams<T> zp, int *__restrict__ err) {
  using V = typename Cx<T>::type;
  constexpr int NTHR = Split<N>::R1 * B;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int m = g.m;
  V *buf = reinterpret_cast<V *>(smem_raw);
  V *tw = buf + m * N * B;
  uint64_t *bar = reinterpret_cast<uint64_t *>(tw + N);
  const int tid = threadIdx.x;
  const int kx0 = blockIdx.x * B, y = blockIdx.y;
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(bar, (uint32_t)(m * N * B * sizeof(V)));
    for (int s = 0; s < m; ++s)
#pragma unroll
      for (int c = 0; c < N; c += kTmaRows) tma_load_3d(buf + s * N * B + c * B, &tm, bar, 2 * kx0, y, s * g.N2 + c);
  }
  for (int q = tid; q < N; q += NTHR) tw[q] = twg[q];
  if (!cta_wait_tile(bar, 0, kMbarPolls, err, 2)) return;
  z_tile<T, MODE, N, B, MS>(g, buf, tw, zp, kx0, y);
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < m; ++s)
#pragma unroll
      for (int c = 0; c < N; c += kTmaRows) tma_store_3d(&tm, buf + s * N * B + c * B, 2 * kx0, y, s * g.N2 + c);
    tma_commit();
    tma_wait_read0();
  }
}

// The z pass from persistent CTAs with two tile buffers: the TMA load of the
// next tile is in flight while the current one is transformed, and the
// store of a tile drains while the next is transformed.  Tiles t =
// blockIdx.x, blockIdx.x + gridDim.x, ... (kx-block t % nkx, ky t / nkx).
template <typename T, int MODE, int N, int B, int MS>
__global__ void __launch_bounds__(Split<N>::R1 * B) k_z_sp(Geo g, const __grid_constant__ CUtensorMap tm,
                                                          const typename Cx<T>::type *__restrict__ twg,
                                                          ZParams<T> zp, int *__restrict__ err) {
  using V = typename Cx<T>::type;
  constexpr int NTHR = Split<N>::R1 * B;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int m = g.m;
  V *bufs[2];
  bufs[0] = reinterpret_cast<V *>(smem_raw);
  bufs[1] = bufs[0] + m * N * B;
  V *tw = bufs[1] + m * N * B;
  uint64_t *bar = reinterpret_cast<uint64_t *>(tw + N);
  const int tid = threadIdx.x;
  const int nkx = (g.Nh + B - 1) / B;
  const int ntile = nkx * g.N1;
  const uint32_t bytes = (uint32_t)(m * N * B * sizeof(V));
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  __syncthreads();
  int t = blockIdx.x;
  if (tid == 0 && t < ntile) {
    mbar_expect_tx(&bar[0], bytes);
    for (int s = 0; s < m; ++s)
#pragma unroll
      for (int c = 0; c < N; c += kTmaRows)
        tma_load_3d(bufs[0] + s * N * B + c * B, &tm, &bar[0], 2 * (t % nkx) * B, t / nkx, s * g.N2 + c);
  }
  for (int q = tid; q < N; q += NTHR) tw[q] = twg[q];
  for (int it = 0; t < ntile; t += gridDim.x, ++it) {
    const int cur = it & 1;
    const int tn = t + gridDim.x;
    if (tid == 0 && tn < ntile) {
      // the other buffer's last store must have read shared memory first
      tma_wait_read0();
      mbar_expect_tx(&bar[cur ^ 1], bytes);
      for (int s = 0; s < m; ++s)
#pragma unroll
        for (int c = 0; c < N; c += kTmaRows)
          tma_load_3d(bufs[cur ^ 1] + s * N * B + c * B, &tm, &bar[cur ^ 1], 2 * (tn % nkx) * B, tn / nkx,
                      s * g.N2 + c);
    }
    const bool ok = mbar_wait(&bar[cur], (uint32_t)((it >> 1) & 1), kMbarPolls);
    if (__syncthreads_or(!ok)) {
      // a CTA-uniform exit: both buffers' loads (this tile's and the
      // prefetch of the next) get one more bounded wait, and the stores
      // drain, before the CTA leaves
      if (tid == 0) {
        atomicExch(err, 2);
        mbar_wait(&bar[cur], (uint32_t)((it >> 1) & 1), kMbarPolls);
        if (tn < ntile) mbar_wait(&bar[cur ^ 1], (uint32_t)(((it + 1) >> 1) & 1), kMbarPolls);
        tma_wait0();
      }
      __syncthreads();
      return;
    }
    const int kx0 = (t % nkx) * B, y = t / nkx;
    z_tile<T, MODE, N, B, MS>(g, bufs[cur], tw, zp, kx0, y);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      for (int s = 0; s < m; ++s)
#pragma unroll
        for (int c = 0; c < N; c += kTmaRows)
          tma_store_3d(&tm, bufs[cur] + s * N * B + c * B, 2 * kx0, y, s * g.N2 + c);
      tma_commit();
    }
  }
  if (tid == 0) tma_wait0();
}

}  // namespace rism
