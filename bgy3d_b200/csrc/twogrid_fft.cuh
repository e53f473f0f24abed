// twogrid_fft.cuh -- the x-axis grid transfers of the two-grid
// preconditioner by FFT, for the row lengths with shape-specialised
// transforms (N0 = 2M).
//
// Restriction of a row x (N0 reals) to Nc coarse points, K = Nc/2:
//   out_i = (s/N0) [X_0 + 2 sum_{0<k<K} Re(e^{2 pi i k i/Nc} X_k) + Re(e^{2 pi i K i/Nc} X_K)],
// X = r2c(x) -- only X_0..X_K are formed after the row transform.
// Prolongation of a coarse row y (Nc reals) with the residual term:
//   out_j = c2r(X)_j - s r_j,  X_k = f_k sum_i y_i e^{-2 pi i k i/Nc},
// f_k = 1/Nc for k < K, 1/(2 Nc) at the Nyquist k = K, X_k = 0 above K.
// Both equal the dense band-limited transfers of twogrid.cuh (the same
// R and P) at about a third of the arithmetic: the row transform is the
// half-length complex FFT of the x passes plus the r2c untangle, and the
// coarse side is a (K+1) x Nc table product.  Transforms run in FP32.
#pragma once
#include "fft_static.cuh"

namespace rism {

template <typename T> __device__ __forceinline__ float2 ld_pair(const T *p);
template <> __device__ __forceinline__ float2 ld_pair<float>(const float *p) {
  return *reinterpret_cast<const float2 *>(p);
}
template <> __device__ __forceinline__ float2 ld_pair<double>(const double *p) {
  const double2 v = *reinterpret_cast<const double2 *>(p);
  return make_float2((float)v.x, (float)v.y);
}

template <int M, int RX> __host__ __device__ constexpr int fx_buf() { return RX * LayRow<M, SplitRow<M>::R2>::RS; }

// Shared memory of the two kernels (bytes) for K = Nc/2: twiddles, the row
// tiles, the coarse-side table, the kept spectrum (and the coarse rows).
template <int M, int RX> inline size_t fx_smem_restrict(int K, int Nc) {
  return sizeof(float2) * (size_t)(M + fx_buf<M, RX>() + (K + 1) * Nc + RX * (K + 1));
}
template <int M, int RX> inline size_t fx_smem_prolong(int K, int Nc) {
  return sizeof(float2) * (size_t)(M + fx_buf<M, RX>() + (K + 1) * Nc + RX * (K + 1)) +
         sizeof(float) * (size_t)RX * Nc;
}

// Vector access of 2 complex values (4 reals) of a row.
template <typename T> struct Quad;
template <> struct Quad<float> {
  using type = float4;
  __device__ __forceinline__ static void split(const float4 &v, float2 &a, float2 &b) {
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
  }
};
template <> struct Quad<double> {
  struct type { double2 a, b; };
  __device__ __forceinline__ static void split(const type &v, float2 &a, float2 &b) {
    a = make_float2((float)v.a.x, (float)v.a.y);
    b = make_float2((float)v.b.x, (float)v.b.y);
  }
};

// out[row][i] (rows x Nc, FP32) = restriction of s * in[row][.] (rows x 2M).
// ctab[k][i] = c_k e^{2 pi i k i / Nc} / N0, c = 1, 2, ..., 2, 1.
// Persistent: each CTA stages the twiddles and the table once and walks
// batches of RX rows with stride gridDim.x; the next batch's rows are loaded
// into registers while the current one is transformed.
template <typename TI, int M, int RX>
__global__ void __launch_bounds__(256) k_restrict_fx(long long rows, int Nc, int K, const TI *__restrict__ in,
                                                     float s, const float2 *__restrict__ post,
                                                     const float2 *__restrict__ twg,
                                                     const float2 *__restrict__ ctab, float *__restrict__ out) {
  using V = float2;
  using Lay = LayRow<M, SplitRow<M>::R2>;
  using Q = typename Quad<TI>::type;
  constexpr int N0 = 2 * M, PER = M / 2, CNT = (RX * PER + 255) / 256;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + M;
  V *C = buf + fx_buf<M, RX>();
  const int K1 = K + 1;
  V *X = C + K1 * Nc;
  const int tid = threadIdx.x;
  const long long nbat = (rows + RX - 1) / RX;
  long long bat = blockIdx.x;
  Q ra[CNT];
#define FX_LOAD_ROWS(BAT)                                                                           \
  {                                                                                                 \
    const long long r0 = (BAT) * RX;                                                                \
    _Pragma("unroll") for (int it = 0; it < CNT; ++it) {                                            \
      const int e = tid + it * 256;                                                                 \
      const int row = e / PER, jj = (e % PER) * 2;                                                  \
      if (e < RX * PER && r0 + row < rows) ra[it] = *reinterpret_cast<const Q *>(in + (r0 + row) * N0 + 2 * jj); \
    }                                                                                               \
  }
  if (bat < nbat) FX_LOAD_ROWS(bat)
  for (int q = tid; q < M; q += 256) tw[q] = twg[q];
  for (int q = tid; q < K1 * Nc; q += 256) C[q] = ctab[q];
  for (; bat < nbat; bat += gridDim.x) {
    const long long row0 = bat * RX;
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * 256;
      if (e >= RX * PER) break;
      const int row = e / PER, jj = (e % PER) * 2;
      V a = make_float2(0.f, 0.f), b = a;
      if (row0 + row < rows) {
        Quad<TI>::split(ra[it], a, b);
        a.x *= s; a.y *= s; b.x *= s; b.y *= s;
      }
      buf[Lay::at(jj, row)] = a;
      buf[Lay::at(jj + 1, row)] = b;
    }
    if (bat + gridDim.x < nbat) FX_LOAD_ROWS(bat + gridDim.x)
    __syncthreads();
    fft2<M, RX, 256, false, false, Lay, SplitRow<M>>(buf, tw);
    for (int e = tid; e < RX * K1; e += 256) {
      const int row = e / K1, k = e - row * K1;
      const V zk = buf[Lay::at(k, row)];
      const V zm = buf[Lay::at(k == 0 ? 0 : M - k, row)];
      V E, O;
      E.x = (zk.x + zm.x) * 0.5f;
      E.y = (zk.y - zm.y) * 0.5f;
      O.x = (zk.y + zm.y) * 0.5f;
      O.y = -(zk.x - zm.x) * 0.5f;
      X[row * K1 + k] = cadd(E, cmul(post[k], O));
    }
    __syncthreads();
    // (K+1) x Nc table product, register-blocked 2 rows x 4 outputs per
    // thread: 6 shared loads per 8 complex products (shared-memory bandwidth
    // bounds this loop)
    {
      const int NQ = (Nc + 3) / 4;
      for (int e = tid; e < (RX / 2) * NQ; e += 256) {
        const int r2 = (e / NQ) * 2, i0 = (e % NQ) * 4;
        float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
        for (int k = 0; k < K1; ++k) {
          const V x0 = X[r2 * K1 + k], x1 = X[(r2 + 1) * K1 + k];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const V c = i0 + q < Nc ? C[k * Nc + i0 + q] : make_float2(0.f, 0.f);
            acc[0][q] = fmaf(c.x, x0.x, fmaf(-c.y, x0.y, acc[0][q]));
            acc[1][q] = fmaf(c.x, x1.x, fmaf(-c.y, x1.y, acc[1][q]));
          }
        }
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          if (row0 + r2 + rr >= rows) continue;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (i0 + q < Nc) out[(row0 + r2 + rr) * Nc + i0 + q] = acc[rr][q];
        }
      }
    }
    __syncthreads();
  }
#undef FX_LOAD_ROWS
}

// out[row][j] (rows x 2M) = prolongation of y[row][.] (rows x Nc, FP32) - s r.
// dtab[i][k] = f_k e^{-2 pi i k i / Nc} (k fastest).  Persistent as
// k_restrict_fx: the next batch's coarse rows and subtracted fine rows are
// in flight while the current batch is transformed.
template <typename TO, typename TR, int M, int RX>
__global__ void __launch_bounds__(256) k_prolong_fx(long long rows, int Nc, int K, const float *__restrict__ y,
                                                    const float2 *__restrict__ post, const float2 *__restrict__ twg,
                                                    const float2 *__restrict__ dtab, const TR *__restrict__ r,
                                                    double s, TO *__restrict__ out) {
  using V = float2;
  using Lay = LayRow<M, SplitRow<M>::R2>;
  using QR = typename Quad<TR>::type;
  constexpr int N0 = 2 * M, H = M / 2 + 1, PER = M / 2, CNT = (RX * PER + 255) / 256;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + M;
  const int K1 = K + 1;
  V *D = buf + fx_buf<M, RX>();
  V *X = D + K1 * Nc;
  float *ys = reinterpret_cast<float *>(X + RX * K1);
  const int tid = threadIdx.x;
  const long long nbat = (rows + RX - 1) / RX;
  const int YC = (RX * Nc + 255) / 256;  // coarse values per thread; Nc < 2M <= 256 keeps it <= RX
  long long bat = blockIdx.x;
  QR rr[CNT], rn[CNT];
  float yv[RX];
#define FX_LOAD(BAT, RR)                                                                            \
  {                                                                                                 \
    const long long r0 = (BAT) * RX;                                                                \
    _Pragma("unroll") for (int it = 0; it < CNT; ++it) {                                            \
      const int e = tid + it * 256;                                                                 \
      const int row = e / PER, jj = (e % PER) * 2;                                                  \
      if (e < RX * PER && r0 + row < rows) RR[it] = *reinterpret_cast<const QR *>(r + (r0 + row) * N0 + 2 * jj); \
    }                                                                                               \
    _Pragma("unroll") for (int q = 0; q < RX; ++q) {                                                \
      const int e = tid + q * 256;                                                                  \
      if (q < YC) yv[q] = (e < RX * Nc && r0 + e / Nc < rows) ? y[r0 * Nc + e] : 0.f;               \
    }                                                                                               \
  }
  if (bat < nbat) FX_LOAD(bat, rr)
  for (int q = tid; q < M; q += 256) tw[q] = twg[q];
  for (int q = tid; q < K1 * Nc; q += 256) D[q] = dtab[q];
  for (; bat < nbat; bat += gridDim.x) {
    const long long row0 = bat * RX;
#pragma unroll
    for (int q = 0; q < RX; ++q) {
      const int e = tid + q * 256;
      if (q < YC && e < RX * Nc) ys[e] = yv[q];
    }
    const bool more = bat + gridDim.x < nbat;
    if (more) FX_LOAD(bat + gridDim.x, rn)
    __syncthreads();
    // Nc x (K+1) table product, register-blocked 2 rows x 3 coefficients
    // per thread: 5 shared loads per 6 complex products
    {
      const int KQ = (K1 + 2) / 3;
      for (int e = tid; e < (RX / 2) * KQ; e += 256) {
        const int r2 = (e / KQ) * 2, k0 = (e % KQ) * 3;
        float ax[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, ay[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        for (int i = 0; i < Nc; ++i) {
          const float v0 = ys[r2 * Nc + i], v1 = ys[(r2 + 1) * Nc + i];
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            const V d = k0 + q < K1 ? D[i * K1 + k0 + q] : make_float2(0.f, 0.f);
            ax[0][q] = fmaf(d.x, v0, ax[0][q]);
            ay[0][q] = fmaf(d.y, v0, ay[0][q]);
            ax[1][q] = fmaf(d.x, v1, ax[1][q]);
            ay[1][q] = fmaf(d.y, v1, ay[1][q]);
          }
        }
#pragma unroll
        for (int rr = 0; rr < 2; ++rr)
#pragma unroll
          for (int q = 0; q < 3; ++q)
            if (k0 + q < K1) X[(r2 + rr) * K1 + k0 + q] = make_float2(ax[rr][q], ay[rr][q]);
      }
    }
    __syncthreads();
    for (int e = tid; e < RX * H; e += 256) {
      const int row = e / H, k = e - row * H;
      V xk = make_float2(0.f, 0.f), xm = make_float2(0.f, 0.f);
      if (k <= K) xk = X[row * K1 + k];
      if (M - k <= K) xm = X[row * K1 + (M - k)];
      if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
      V Aa, Dd;
      Aa.x = xk.x + xm.x; Aa.y = xk.y - xm.y;
      Dd.x = xk.x - xm.x; Dd.y = xk.y + xm.y;
      const V Pp = cmul(Dd, cconj(post[k]));
      V zk, zm;
      zk.x = Aa.x - Pp.y; zk.y = Aa.y + Pp.x;
      zm.x = Aa.x + Pp.y; zm.y = -(Aa.y - Pp.x);
      buf[Lay::at(k, row)] = zk;
      if (k != 0 && M - k != k) buf[Lay::at(M - k, row)] = zm;
    }
    __syncthreads();
    fft2<M, RX, 256, true, false, Lay, SplitRow<M>>(buf, tw);
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * 256;
      if (e >= RX * PER) break;
      const int row = e / PER, jj = (e % PER) * 2;
      if (row0 + row >= rows) continue;
      V ra, rb;
      Quad<TR>::split(rr[it], ra, rb);
      const V za = buf[Lay::at(jj, row)], zb = buf[Lay::at(jj + 1, row)];
      TO *o = out + (row0 + row) * N0 + 2 * jj;
      // the subtracted term in the output precision (r kept exact for FP64)
      const TR *rx = r + (row0 + row) * N0 + 2 * jj;
      if (sizeof(TR) == 8) {
        o[0] = (TO)((double)za.x - s * (double)rx[0]);
        o[1] = (TO)((double)za.y - s * (double)rx[1]);
        o[2] = (TO)((double)zb.x - s * (double)rx[2]);
        o[3] = (TO)((double)zb.y - s * (double)rx[3]);
      } else {
        const float sf = (float)s;
        o[0] = (TO)(za.x - sf * ra.x);
        o[1] = (TO)(za.y - sf * ra.y);
        o[2] = (TO)(zb.x - sf * rb.x);
        o[3] = (TO)(zb.y - sf * rb.y);
      }
    }
    if (more) {
#pragma unroll
      for (int it = 0; it < CNT; ++it) rr[it] = rn[it];
    }
    __syncthreads();
  }
#undef FX_LOAD
}

}  // namespace rism

namespace rism {

// ---- both sides by FFT: the coarse side as a packed row transform of
// length Nc = 2 MC instead of the (K+1) x Nc table product (K = MC).
//
// Restriction: out = c2r_Nc(X_0..X_K) / N0 (Im X_0, Im X_K dropped, as the
// table's c_k weights do), i.e. the K+1 kept coefficients are packed into
// MC complex values and transformed by the MC-point inverse FFT; the packed
// result z_j = out_{2j} + i out_{2j+1}.
// Prolongation: X_k = f_k r2c_Nc(y)_k from the MC-point forward FFT of the
// coarse row and its untangle, then the fine packed c2r as before.
// twc / postc: the twiddles of the MC-point transform and exp(-2 pi i k / Nc),
// k in [0, MC] (the coarse grid's own x tables).  The coarse row tile
// aliases the fine one (it is only live while the fine one is not).
template <int M, int MC, int RX> __host__ __device__ constexpr int fx2_words() {
  return M + fx_buf<M, RX>() + RX * (MC + 1) + MC;
}
template <int M, int MC, int RX> inline size_t fx2_smem() { return sizeof(float2) * (size_t)fx2_words<M, MC, RX>(); }

// z-pack of a Hermitian half spectrum X_0..X_K (row stride K1) for the packed
// c2r of length 2 MM (K >= MM: only X_0..X_MM are read; K < MM: zero above
// K).  Writes the MM packed values of every row into buf (layout L).
template <int MM, int RX, class L>
__device__ __forceinline__ void fx_pack_c2r(const float2 *X, int K, int K1, const float2 *post, float2 *buf) {
  constexpr int H = MM / 2 + 1;
  for (int e = threadIdx.x; e < RX * H; e += 256) {
    const int row = e / H, k = e - row * H;
    float2 xk = make_float2(0.f, 0.f), xm = make_float2(0.f, 0.f);
    if (k <= K) xk = X[row * K1 + k];
    if (MM - k <= K) xm = X[row * K1 + (MM - k)];
    if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
    float2 Aa, Dd;
    Aa.x = xk.x + xm.x; Aa.y = xk.y - xm.y;
    Dd.x = xk.x - xm.x; Dd.y = xk.y + xm.y;
    const float2 Pp = cmul(Dd, cconj(post[k]));
    float2 zk, zm;
    zk.x = Aa.x - Pp.y; zk.y = Aa.y + Pp.x;
    zm.x = Aa.x + Pp.y; zm.y = -(Aa.y - Pp.x);
    buf[L::at(k, row)] = zk;
    if (k != 0 && MM - k != k) buf[L::at(MM - k, row)] = zm;
  }
}

// 128-point half rows at 3 CTAs per SM (80 registers, no spills; the
// unbounded choice of 128 allows 2): the batches are latency chains, so
// resident CTAs set the throughput.
template <typename TI, int M, int MC, int RX>
__global__ void __launch_bounds__(256, M == 128 ? 3 : 1) k_restrict_fx2(long long rows, const TI *__restrict__ in, float s,
                                                      const float2 *__restrict__ post, const float2 *__restrict__ twg,
                                                      const float2 *__restrict__ postc,
                                                      const float2 *__restrict__ twcg, float *__restrict__ out) {
  using V = float2;
  using Lay = LayRow<M, SplitRow<M>::R2>;
  using LayC = LayRow<MC, SplitRow<MC>::R2>;
  using Q = typename Quad<TI>::type;
  static_assert(MC < M && fx_buf<MC, RX>() <= fx_buf<M, RX>(), "coarse row tile must fit the fine one");
  constexpr int N0 = 2 * M, Nc = 2 * MC, K = MC, K1 = MC + 1;
  constexpr int PER = M / 2, CNT = (RX * PER + 255) / 256;
  constexpr int PC = MC / 2;  // output float4 per row
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + M;
  V *X = buf + fx_buf<M, RX>();
  V *twc = X + RX * K1;
  const int tid = threadIdx.x;
  const long long nbat = (rows + RX - 1) / RX;
  const float inv_n0 = 1.0f / (float)N0;
  long long bat = blockIdx.x;
  Q ra[CNT];
#define FX2_LOAD_ROWS(BAT)                                                                          \
  {                                                                                                 \
    const long long r0 = (BAT) * RX;                                                                \
    _Pragma("unroll") for (int it = 0; it < CNT; ++it) {                                            \
      const int e = tid + it * 256;                                                                 \
      const int row = e / PER, jj = (e % PER) * 2;                                                  \
      if (e < RX * PER && r0 + row < rows) ra[it] = *reinterpret_cast<const Q *>(in + (r0 + row) * N0 + 2 * jj); \
    }                                                                                               \
  }
  if (bat < nbat) FX2_LOAD_ROWS(bat)
  for (int q = tid; q < M; q += 256) tw[q] = twg[q];
  for (int q = tid; q < MC; q += 256) twc[q] = twcg[q];
  for (; bat < nbat; bat += gridDim.x) {
    const long long row0 = bat * RX;
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * 256;
      if (e >= RX * PER) break;
      const int row = e / PER, jj = (e % PER) * 2;
      V a = make_float2(0.f, 0.f), b = a;
      if (row0 + row < rows) {
        Quad<TI>::split(ra[it], a, b);
        a.x *= s; a.y *= s; b.x *= s; b.y *= s;
      }
      buf[Lay::at(jj, row)] = a;
      buf[Lay::at(jj + 1, row)] = b;
    }
    if (bat + gridDim.x < nbat) FX2_LOAD_ROWS(bat + gridDim.x)
    __syncthreads();
    fft2<M, RX, 256, false, false, Lay, SplitRow<M>>(buf, tw);
    for (int e = tid; e < RX * K1; e += 256) {
      const int row = e / K1, k = e - row * K1;
      const V zk = buf[Lay::at(k, row)];
      const V zm = buf[Lay::at(k == 0 ? 0 : M - k, row)];
      V E, O;
      E.x = (zk.x + zm.x) * 0.5f;
      E.y = (zk.y - zm.y) * 0.5f;
      O.x = (zk.y + zm.y) * 0.5f;
      O.y = -(zk.x - zm.x) * 0.5f;
      X[row * K1 + k] = cadd(E, cmul(post[k], O));
    }
    __syncthreads();
    fx_pack_c2r<MC, RX, LayC>(X, K, K1, postc, buf);
    __syncthreads();
    fft2<MC, RX, 256, true, false, LayC, SplitRow<MC>>(buf, twc);
    for (int e = tid; e < RX * PC; e += 256) {
      const int row = e / PC, jj = (e - row * PC) * 2;
      if (row0 + row >= rows) continue;
      const V za = buf[LayC::at(jj, row)], zb = buf[LayC::at(jj + 1, row)];
      *reinterpret_cast<float4 *>(out + (row0 + row) * Nc + 2 * jj) =
          make_float4(za.x * inv_n0, za.y * inv_n0, zb.x * inv_n0, zb.y * inv_n0);
    }
    __syncthreads();
  }
#undef FX2_LOAD_ROWS
}

// 128-point half rows (the 256^3 grid) at 3 CTAs per SM: at the compiler's
// unbounded choice of 128 registers only 2 fit; the bound costs a few spilled
// words there (more at 256-point rows, which keep the unbounded choice)
template <typename TO, typename TR, int M, int MC, int RX>
__global__ void __launch_bounds__(256, M == 128 ? (RX >= 32 ? 2 : 3) : 1) k_prolong_fx2(long long rows, const float *__restrict__ y,
                                                     const float2 *__restrict__ post, const float2 *__restrict__ twg,
                                                     const float2 *__restrict__ postc,
                                                     const float2 *__restrict__ twcg, const TR *__restrict__ r,
                                                     double s, TO *__restrict__ out) {
  using V = float2;
  using Lay = LayRow<M, SplitRow<M>::R2>;
  using LayC = LayRow<MC, SplitRow<MC>::R2>;
  using QR = typename Quad<TR>::type;
  static_assert(MC < M && fx_buf<MC, RX>() <= fx_buf<M, RX>(), "coarse row tile must fit the fine one");
  constexpr int N0 = 2 * M, Nc = 2 * MC, K = MC, K1 = MC + 1;
  constexpr int PER = M / 2, CNT = (RX * PER + 255) / 256;
  constexpr int YC = (RX * MC + 255) / 256;  // coarse pairs per thread
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V *tw = reinterpret_cast<V *>(smem_raw);
  V *buf = tw + M;
  V *X = buf + fx_buf<M, RX>();
  V *twc = X + RX * K1;
  const int tid = threadIdx.x;
  const long long nbat = (rows + RX - 1) / RX;
  const float fk = 1.0f / (float)Nc;
  long long bat = blockIdx.x;
  QR rr[CNT], rn[CNT];
  V yv[YC];
#define FX2_LOAD(BAT, RR)                                                                           \
  {                                                                                                 \
    const long long r0 = (BAT) * RX;                                                                \
    _Pragma("unroll") for (int it = 0; it < CNT; ++it) {                                            \
      const int e = tid + it * 256;                                                                 \
      const int row = e / PER, jj = (e % PER) * 2;                                                  \
      if (e < RX * PER && r0 + row < rows) RR[it] = *reinterpret_cast<const QR *>(r + (r0 + row) * N0 + 2 * jj); \
    }                                                                                               \
    _Pragma("unroll") for (int q = 0; q < YC; ++q) {                                                \
      const int e = tid + q * 256;                                                                  \
      yv[q] = (e < RX * MC && r0 + e / MC < rows) ? *reinterpret_cast<const float2 *>(y + r0 * Nc + 2 * e) \
                                                 : make_float2(0.f, 0.f);                          \
    }                                                                                               \
  }
  if (bat < nbat) FX2_LOAD(bat, rr)
  for (int q = tid; q < M; q += 256) tw[q] = twg[q];
  for (int q = tid; q < MC; q += 256) twc[q] = twcg[q];
  for (; bat < nbat; bat += gridDim.x) {
    const long long row0 = bat * RX;
#pragma unroll
    for (int q = 0; q < YC; ++q) {
      const int e = tid + q * 256;
      if (e < RX * MC) buf[LayC::at(e % MC, e / MC)] = yv[q];
    }
    const bool more = bat + gridDim.x < nbat;
    if (more) FX2_LOAD(bat + gridDim.x, rn)
    __syncthreads();
    fft2<MC, RX, 256, false, false, LayC, SplitRow<MC>>(buf, twc);
    // untangle to the Nc-point r2c, weights f_k (1/Nc, half at the Nyquist K)
    for (int e = tid; e < RX * K1; e += 256) {
      const int row = e / K1, k = e - row * K1;
      V xk;
      if (k == K) {
        const V z0 = buf[LayC::at(0, row)];
        xk = make_float2((z0.x - z0.y) * 0.5f * fk, 0.f);
      } else {
        const V zk = buf[LayC::at(k, row)];
        const V zm = buf[LayC::at(k == 0 ? 0 : MC - k, row)];
        V E, O;
        E.x = (zk.x + zm.x) * 0.5f;
        E.y = (zk.y - zm.y) * 0.5f;
        O.x = (zk.y + zm.y) * 0.5f;
        O.y = -(zk.x - zm.x) * 0.5f;
        xk = cadd(E, cmul(postc[k], O));
        xk.x *= fk; xk.y *= fk;
      }
      X[row * K1 + k] = xk;
    }
    __syncthreads();
    fx_pack_c2r<M, RX, Lay>(X, K, K1, post, buf);
    __syncthreads();
    fft2<M, RX, 256, true, false, Lay, SplitRow<M>>(buf, tw);
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * 256;
      if (e >= RX * PER) break;
      const int row = e / PER, jj = (e % PER) * 2;
      if (row0 + row >= rows) continue;
      V ra, rb;
      Quad<TR>::split(rr[it], ra, rb);
      const V za = buf[Lay::at(jj, row)], zb = buf[Lay::at(jj + 1, row)];
      TO *o = out + (row0 + row) * N0 + 2 * jj;  // 4 consecutive outputs, 4-element aligned
      const TR *rx = r + (row0 + row) * N0 + 2 * jj;
      if constexpr (sizeof(TR) == 8) {
        // the subtracted term in the output precision (r kept exact for FP64)
        const double2 r01 = *reinterpret_cast<const double2 *>(rx), r23 = *reinterpret_cast<const double2 *>(rx + 2);
        const double o0 = (double)za.x - s * r01.x, o1 = (double)za.y - s * r01.y;
        const double o2 = (double)zb.x - s * r23.x, o3 = (double)zb.y - s * r23.y;
        if constexpr (sizeof(TO) == 8) {
          *reinterpret_cast<double2 *>(o) = make_double2(o0, o1);
          *reinterpret_cast<double2 *>(o + 2) = make_double2(o2, o3);
        } else {
          o[0] = (TO)o0; o[1] = (TO)o1; o[2] = (TO)o2; o[3] = (TO)o3;
        }
      } else {
        const float sf = (float)s;
        const float o0 = za.x - sf * ra.x, o1 = za.y - sf * ra.y, o2 = zb.x - sf * rb.x, o3 = zb.y - sf * rb.y;
        if constexpr (sizeof(TO) == 4) {
          *reinterpret_cast<float4 *>(o) = make_float4(o0, o1, o2, o3);
        } else {
          o[0] = (TO)o0; o[1] = (TO)o1; o[2] = (TO)o2; o[3] = (TO)o3;
        }
      }
    }
    if (more) {
#pragma unroll
      for (int it = 0; it < CNT; ++it) rr[it] = rn[it];
    }
    __syncthreads();
  }
#undef FX2_LOAD
}

}  // namespace rism
