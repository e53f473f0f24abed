// coarse_pk.cuh -- the coarse solve of the two-grid preconditioner as ONE
// persistent cooperative kernel (sm_100a).
//
// J_H^-1 r is k steps of GMRES from zero on the coarse problem (a 64^3 grid
// at the 256^3 workload: every vector, the basis and the work buffer stay in
// the 126 MB L2).  Launched step by step that is 8 kernels per step -- five
// FFT passes, a dot sweep, an update sweep, a scaling -- each a few
// microseconds of L2 traffic behind a launch and a grid drain.  Here the
// whole solve is one cooperative grid whose CTAs walk the same work items
// as the step-by-step passes and meet at a grid barrier between phases:
//
//   P0   |r|^2 partials                                        | barrier
//   per step j = 0 .. k-1:
//   XF   V_j -= sum_{i<j} c_i V_i (the Gram-Schmidt update of step j-1,
//        with its |.|^2 partials), then c'_H V_j and the r2c along x  | barrier
//   Y    forward along y                                       | barrier
//   Z    along z, the OZ contraction, inverse along z          | barrier
//   YI   inverse along y                                       | barrier
//   XI   c2r along x: V_{j+1} = (X / N - V_j) / s_j = J (V_j / s_j), with
//        the dot partials <V_i, V_{j+1}>, i <= j                | barrier
//   then the update of V_k with its norm (barrier), the (k+1) x k least
//   squares, and out = sum_j y_j V_j / s_j.
//
// The basis is kept unnormalised (V_j holds s_j times the unit vector, s_j
// its norm): the scaling sweep disappears into the factors the next passes
// apply anyway.  Every CTA sums the block partials of a reduction itself,
// in one fixed order, so all CTAs hold bitwise the same Hessenberg matrix
// and norms without a further barrier; partial buffers alternate so that no
// CTA overwrites partials another may still be summing.
//
// The grid barrier is a counter in global memory (zeroed before the launch)
// that every CTA's thread 0 increments (release) and polls (acquire) with a
// bounded number of polls; on a timeout, or when another CTA has reported
// one, the CTA records the error and leaves, so a failure ends the kernel
// with a status instead of a hang.  The launch is cooperative, so the CTAs
// are co-resident by construction.  No data written inside the kernel is
// read through the non-coherent path (no __restrict__ const on W or V).
#pragma once
#include "kernels_static.cuh"
#include "krylov.cuh"

namespace rism {

constexpr int kPkThreads = 256;
constexpr int kPkMaxSteps = 16;        // coarse GMRES steps (the basis holds k + 1 vectors)
constexpr uint32_t kGridPolls = 1u << 22;  // bounded grid-barrier wait (seconds with the back-off)
constexpr int kPkErr = 4;              // d_err code of a grid-barrier timeout

struct PkArgs {
  Geo g;                 // coarse grid: N0 = 2M, N1 = N2 = N, m <= 3
  float2 *W;             // complex work buffer [m][N2][N1][Nhp]
  float *V[kPkMaxSteps + 1];  // basis slots; V[0] holds r on entry
  const float *d;        // coarse closure slope c'_H
  float *out;            // sum_j y_j V_j / s_j = J_H^-1 r + r
  const float2 *post;    // r2c untangling weights along x
  const float2 *twx, *twy, *twz;
  ZParams<float> zp;     // Jacobian form: chi - 1 tables only
  double *pdot;          // [grid][kVecMax] dot partials
  double *pnrm;          // [2][grid] norm partials (alternating)
  double *H;             // [k][k+1] Hessenberg columns (CTA 0 writes them out)
  double *aux;           // [k + 2]: s_0, then y (CTA 0)
  unsigned *bar;         // barrier counter, zero at launch
  int *err;              // set to kPkErr on a barrier timeout
  int k;                 // GMRES steps, 1 .. kPkMaxSteps
  unsigned long long *trace;  // diagnostics, or null: %globaltimer at the start and at every barrier (CTA 0)
  unsigned long long *trace_cta;  // diagnostics, or null: [barrier][2][grid] arrival / release of every CTA
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid barrier number `gen` (1, 2, ...): done when the counter reaches
// gen * gridDim.x.  CTA-uniform result; false: leave the kernel.
__device__ __forceinline__ bool grid_sync(unsigned *bar, unsigned gen, int *err,
                                          unsigned long long *trace = nullptr,
                                          unsigned long long *trace_cta = nullptr) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (trace_cta) trace_cta[(size_t)(gen - 1) * 2 * gridDim.x + blockIdx.x] = global_ns();
    // arrive with release semantics (the CTA's writes, ordered before this
    // thread by the barrier above, become visible first), then poll with
    // acquire loads: the first load that sees every arrival orders all later
    // reads of the CTA (through the barrier below) after the other CTAs' writes
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    const unsigned target = gen * gridDim.x;
    uint32_t polls = 0;
    while (ld_acquire_gpu(bar) < target) {
      if (++polls > kGridPolls || *reinterpret_cast<volatile int *>(err) != 0) {
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    if (!ok) atomicCAS(err, 0, kPkErr);
    s_ok = ok;
    if (trace && blockIdx.x == 0) trace[gen] = global_ns();
    if (trace_cta) trace_cta[(size_t)(gen - 1) * 2 * gridDim.x + gridDim.x + blockIdx.x] = global_ns();
  }
  __syncthreads();
  return s_ok != 0;
}

// out[v] = sum_{b < nb} part[b * stride + v], v < nv (nv <= 32), by the whole
// CTA in a fixed order (identical in every CTA); out in shared memory.
__device__ __forceinline__ void pk_sum_partials(const double *part, int stride, int nb, int nv, double *out) {
  __shared__ double red[kPkThreads];
  int lanes = 1;
  while (lanes < nv) lanes <<= 1;
  const int groups = kPkThreads / lanes;
  const int v = threadIdx.x % lanes, q = threadIdx.x / lanes;
  double s = 0.0;
  if (v < nv) {
#pragma unroll 4
    for (int b = q; b < nb; b += groups) s += part[(long long)b * stride + v];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  // pairwise over the groups (slot q * lanes + v keeps v): log2(groups)
  // steps instead of a chain of `groups` dependent adds
  for (int stride = kPkThreads / 2; stride >= lanes; stride >>= 1) {
    if ((int)threadIdx.x < stride) red[threadIdx.x] += red[threadIdx.x + stride];
    __syncthreads();
  }
  if ((int)threadIdx.x < nv) out[threadIdx.x] = red[threadIdx.x];
  __syncthreads();
}

// Block sum of a per-thread double into part[blockIdx.x] (thread 0 writes).
__device__ __forceinline__ void pk_block_sum(double s, double *part) {
  __shared__ double sm[kPkThreads / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sm[wid] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kPkThreads / 32; ++w) t += sm[w];
    part[blockIdx.x] = t;
  }
}

// The split of the x-phase transforms (measured: the larger first radix of
// Split beats SplitRow at 48-row items of 32-point rows, and ties with it at
// the plane form's 64-row items).
template <int M> using PkSplit = Split<M>;

// Rows of the x phases per work item: about one item per CTA of a 2 x 148
// grid for m = 3, a multiple of 8, at most 4 float4 of a vector per thread.
template <int M> __host__ __device__ constexpr int pk_rx() {
  constexpr int want = ((12 * M * M + 295) / 296 + 7) / 8 * 8;
  constexpr int cap = (2048 / M) / 8 * 8;
  return want < cap ? want : cap;
}

// Basis vectors whose loads a thread keeps in flight together (CNT float4
// of each).
template <int CNT> __host__ __device__ constexpr int pk_group() { return CNT <= 2 ? 4 : 2; }

// The column tile of the plane phases: [N][M + 2] complex (y, kx), the row
// stride of W (Nhp = M + 2 for the even M here), after the row tile.
template <int M> __host__ __device__ constexpr int pk_ncp() { return M + 2; }

// XF: V_j -= sum_{i<nu} cf_i V_i (nu = 0: no update) with |V_j|^2 into nrm2;
// then, if fft, c'_H V_j and the r2c along x into W.  PLANE (RX = N, the
// rows of one (site, z) plane per item): the spectrum goes into the column
// tile, is transformed along y as well, and the plane is stored to W whole.
template <int M, int RX = pk_rx<M>(), bool PLANE = false, int N = RX>
__device__ __forceinline__ void pk_xf(const PkArgs &a, float *const *V, int j, int nu, const float *cf, bool fft,
                                      float2 *buf, const float2 *tw, const float2 *twy, double &nrm2) {
  static_assert(!PLANE || RX == N, "a plane item holds the N rows of one (site, z) plane");
  using Lay = LayRow<M, PkSplit<M>::R2>;
  constexpr int NCP = pk_ncp<M>();
  float2 *T = buf + RX * Lay::RS;  // PLANE: the column tile
  constexpr int PER_ROW = M / 2;  // float4 per row (two complex values)
  constexpr int CNT = (RX * PER_ROW + kPkThreads - 1) / kPkThreads;
  constexpr int H = M / 2 + 1;
  const int tid = threadIdx.x;
  const int rows_total = a.g.m * a.g.N1 * a.g.N2;
  const int nitems = (rows_total + RX - 1) / RX;
  float *w = V[j];
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int row0 = item * RX;
    float4 x[CNT];
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * kPkThreads;
      const int row = e / PER_ROW, jj = (e % PER_ROW) * 2;
      x[it] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (e < RX * PER_ROW && row0 + row < rows_total)
        x[it] = *reinterpret_cast<const float4 *>(w + (long long)(row0 + row) * a.g.N0 + 2 * jj);
    }
    if (nu > 0) {
      // the basis vectors in groups, all loads of a group in flight
      constexpr int GV = pk_group<CNT>();
      for (int i0 = 0; i0 < nu; i0 += GV) {
        float4 b[GV][CNT];
#pragma unroll
        for (int u = 0; u < GV; ++u)
#pragma unroll
          for (int it = 0; it < CNT; ++it) {
            const int e = tid + it * kPkThreads;
            const int row = e / PER_ROW, jj = (e % PER_ROW) * 2;
            if (i0 + u < nu && e < RX * PER_ROW && row0 + row < rows_total)
              b[u][it] = *reinterpret_cast<const float4 *>(V[i0 + u] + (long long)(row0 + row) * a.g.N0 + 2 * jj);
            else
              b[u][it] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
#pragma unroll
        for (int u = 0; u < GV; ++u) {
          const float c = i0 + u < nu ? cf[i0 + u] : 0.f;
#pragma unroll
          for (int it = 0; it < CNT; ++it) {
            x[it].x -= c * b[u][it].x;
            x[it].y -= c * b[u][it].y;
            x[it].z -= c * b[u][it].z;
            x[it].w -= c * b[u][it].w;
          }
        }
      }
#pragma unroll
      for (int it = 0; it < CNT; ++it) {
        const int e = tid + it * kPkThreads;
        const int row = e / PER_ROW, jj = (e % PER_ROW) * 2;
        if (e < RX * PER_ROW && row0 + row < rows_total) {
          *reinterpret_cast<float4 *>(w + (long long)(row0 + row) * a.g.N0 + 2 * jj) = x[it];
          nrm2 += (double)(x[it].x * x[it].x + x[it].y * x[it].y + x[it].z * x[it].z + x[it].w * x[it].w);
        }
      }
    }
    if (!fft) continue;
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * kPkThreads;
      if (e >= RX * PER_ROW) break;
      const int row = e / PER_ROW, jj = (e % PER_ROW) * 2;
      float2 z0 = make_float2(0.f, 0.f), z1 = make_float2(0.f, 0.f);
      if (row0 + row < rows_total) {
        const float4 dd = *reinterpret_cast<const float4 *>(a.d + (long long)(row0 + row) * a.g.N0 + 2 * jj);
        z0 = make_float2(dd.x * x[it].x, dd.y * x[it].y);
        z1 = make_float2(dd.z * x[it].z, dd.w * x[it].w);
      }
      buf[Lay::at(jj, row)] = z0;
      buf[Lay::at(jj + 1, row)] = z1;
    }
    __syncthreads();
    fft2<M, RX, kPkThreads, false, false, Lay, PkSplit<M>>(buf, tw);
    for (int e = tid; e < RX * H; e += kPkThreads) {
      const int row = e / H, kk = e % H;
      const int grow = row0 + row;
      if (grow >= rows_total) continue;
      const float2 zk = buf[Lay::at(kk, row)];
      const float2 zm = buf[Lay::at(kk == 0 ? 0 : M - kk, row)];
      float2 E, O;
      E.x = (zk.x + zm.x) * 0.5f;
      E.y = (zk.y - zm.y) * 0.5f;
      O.x = (zk.y + zm.y) * 0.5f;
      O.y = -(zk.x - zm.x) * 0.5f;
      const float2 wO = cmul(a.post[kk], O);
      float2 *row_out = PLANE ? T + row * NCP : a.W + (long long)grow * a.g.Nhp;
      row_out[kk] = cadd(E, wO);
      if (M - kk != kk) row_out[M - kk] = cconj(csub(E, wO));
    }
    __syncthreads();  // buf is refilled by the next item
    if constexpr (PLANE) {
      fft2g<N, M + 1, kPkThreads, false, true, LayCol<N, NCP>, SplitSq<N>>(T, twy, tid, true);
      float4 *dst = reinterpret_cast<float4 *>(a.W + (long long)item * N * NCP);
      const float4 *src = reinterpret_cast<const float4 *>(T);
      for (int e = tid; e < N * NCP / 2; e += kPkThreads) dst[e] = src[e];
      __syncthreads();  // T is refilled by the next item
    }
  }
}

// XI: V_{j+1} = sc X - sub V_j (X the c2r of W along x), with the dots
// <V_i, V_{j+1}>, i <= j, summed per warp into sdot[i][warp] (shared, zeroed
// by the caller).  PLANE: the item's plane of W is loaded whole into the
// column tile and transformed back along y first.
template <int M, int RX = pk_rx<M>(), bool PLANE = false, int N = RX>
__device__ __forceinline__ void pk_xi(const PkArgs &a, float *const *V, int j, float sc, float sub, float2 *buf,
                                      const float2 *tw, const float2 *twy, double (*sdot)[kPkThreads / 32]) {
  static_assert(!PLANE || RX == N, "a plane item holds the N rows of one (site, z) plane");
  using Lay = LayRow<M, PkSplit<M>::R2>;
  constexpr int NCP = pk_ncp<M>();
  float2 *T = buf + RX * Lay::RS;  // PLANE: the column tile
  constexpr int PER_ROW = M / 2;
  constexpr int CNT = (RX * PER_ROW + kPkThreads - 1) / kPkThreads;
  constexpr int GV = pk_group<CNT>();
  constexpr int H = M / 2 + 1;
  const int tid = threadIdx.x;
  const int lane = tid & 31, wid = tid >> 5;
  const int rows_total = a.g.m * a.g.N1 * a.g.N2;
  const int nitems = (rows_total + RX - 1) / RX;
  const float *vin = V[j];
  float *vout = V[j + 1];
  const int nv = j + 1;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int row0 = item * RX;
    float4 rin[CNT];
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * kPkThreads;
      const int row = e / PER_ROW, jj = (e % PER_ROW) * 2;
      if (e < RX * PER_ROW && row0 + row < rows_total)
        rin[it] = *reinterpret_cast<const float4 *>(vin + (long long)(row0 + row) * a.g.N0 + 2 * jj);
    }
    if constexpr (PLANE) {
      const float4 *src = reinterpret_cast<const float4 *>(a.W + (long long)item * N * NCP);
      float4 *dst = reinterpret_cast<float4 *>(T);
      for (int e = tid; e < N * NCP / 2; e += kPkThreads) dst[e] = src[e];
      __syncthreads();
      fft2g<N, M + 1, kPkThreads, true, true, LayCol<N, NCP>, SplitSq<N>>(T, twy, tid, true);
    }
    for (int e = tid; e < RX * H; e += kPkThreads) {
      const int row = e / H, kk = e % H;
      const int grow = row0 + row;
      float2 zk = make_float2(0.f, 0.f), zm = make_float2(0.f, 0.f);
      if (grow < rows_total) {
        const float2 *row_in = PLANE ? T + row * NCP : a.W + (long long)grow * a.g.Nhp;
        float2 xk = row_in[kk];
        float2 xm = row_in[M - kk];
        if (kk == 0) { xk.y = 0.f; xm.y = 0.f; }  // c2r reads only Re X_0, Re X_{N0/2}
        float2 Aa, D;
        Aa.x = xk.x + xm.x; Aa.y = xk.y - xm.y;
        D.x = xk.x - xm.x;  D.y = xk.y + xm.y;
        const float2 Pp = cmul(D, cconj(a.post[kk]));
        zk.x = Aa.x - Pp.y; zk.y = Aa.y + Pp.x;
        zm.x = Aa.x + Pp.y; zm.y = -(Aa.y - Pp.x);
      }
      buf[Lay::at(kk, row)] = zk;
      if (kk != 0 && M - kk != kk) buf[Lay::at(M - kk, row)] = zm;
    }
    __syncthreads();
    fft2<M, RX, kPkThreads, true, false, Lay, PkSplit<M>>(buf, tw);
    float4 o[CNT];
#pragma unroll
    for (int it = 0; it < CNT; ++it) {
      const int e = tid + it * kPkThreads;
      const int row = e / PER_ROW, jj = (e % PER_ROW) * 2;
      o[it] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (e < RX * PER_ROW && row0 + row < rows_total) {
        const float2 z0 = buf[Lay::at(jj, row)], z1 = buf[Lay::at(jj + 1, row)];
        o[it] = make_float4(z0.x * sc - sub * rin[it].x, z0.y * sc - sub * rin[it].y, z1.x * sc - sub * rin[it].z,
                            z1.y * sc - sub * rin[it].w);
        *reinterpret_cast<float4 *>(vout + (long long)(row0 + row) * a.g.N0 + 2 * jj) = o[it];
      }
    }
    // dots against the basis, GV vectors' loads in flight at a time; each
    // group reduced over the warp (lane 0 adds it to the warp's slot)
    for (int i0 = 0; i0 < nv; i0 += GV) {
      float4 b[GV][CNT];
#pragma unroll
      for (int u = 0; u < GV; ++u)
#pragma unroll
        for (int it = 0; it < CNT; ++it) {
          const int e = tid + it * kPkThreads;
          const int row = e / PER_ROW, jj = (e % PER_ROW) * 2;
          if (i0 + u < nv && e < RX * PER_ROW && row0 + row < rows_total)
            b[u][it] = *reinterpret_cast<const float4 *>(V[i0 + u] + (long long)(row0 + row) * a.g.N0 + 2 * jj);
          else
            b[u][it] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
      for (int u = 0; u < GV; ++u) {
        double d = 0.0;
#pragma unroll
        for (int it = 0; it < CNT; ++it)
          d += (double)(o[it].x * b[u][it].x + o[it].y * b[u][it].y + o[it].z * b[u][it].z + o[it].w * b[u][it].w);
        for (int q = 16; q > 0; q >>= 1) d += __shfl_xor_sync(0xffffffffu, d, q);
        if (lane == 0 && i0 + u < nv) sdot[i0 + u][wid] += d;
      }
    }
    __syncthreads();
  }
}

// Y (INV: inverse): [N][16] column tiles (kx block, z, site), groups of
// R1 * 16 threads, several tiles per CTA at once.
template <int N, bool INV>
__device__ __forceinline__ void pk_y(const PkArgs &a, float2 *smem, const float2 *tw) {
  constexpr int B = 16;
  constexpr int NG = Split<N>::R1 * B;
  constexpr int GPC = kPkThreads / NG;
  static_assert(GPC >= 1, "a y tile needs at most one CTA of threads");
  const Geo &g = a.g;
  const int nkx = (g.Nh + B - 1) / B;
  const int ntile = nkx * g.N2 * g.m;
  const int grp = threadIdx.x / NG, tid = threadIdx.x % NG;
  const bool ing = grp < GPC;
  float2 *buf = smem + (ing ? grp : 0) * N * B;
  for (int base = blockIdx.x * GPC; base < ntile; base += gridDim.x * GPC) {
    const int t = base + grp;
    const bool act = ing && t < ntile;
    const int tt = act ? t : 0;
    const int kx0 = (tt % nkx) * B, rest = tt / nkx;  // rest = site * N2 + z
    float2 *plane = a.W + (long long)rest * g.N1 * g.Nhp;
    if (act) {
      for (int e = tid; e < N * (B / 2); e += NG) {
        const int y = e / (B / 2), b2 = (e % (B / 2)) * 2;
        if (kx0 + b2 < g.Nhp)  // Nhp is even: the pair lies inside the row
          *reinterpret_cast<float4 *>(buf + y * B + b2) =
              *reinterpret_cast<const float4 *>(plane + (long long)y * g.Nhp + kx0 + b2);
      }
    }
    __syncthreads();
    fft2g<N, B, NG, INV, true, LayCol<N, B>>(buf, tw, tid, act);
    if (act) {
      for (int e = tid; e < N * (B / 2); e += NG) {
        const int y = e / (B / 2), b2 = (e % (B / 2)) * 2;
        if (kx0 + b2 < g.Nhp)
          *reinterpret_cast<float4 *>(plane + (long long)y * g.Nhp + kx0 + b2) =
              *reinterpret_cast<const float4 *>(buf + y * B + b2);
      }
    }
    __syncthreads();
  }
}

// Z: the three site tiles [N][4] of one (kx block, ky) transformed as one
// 12-column tile, the OZ contraction, the inverse.  The z transforms split
// N = R1 R2 with R1 about sqrt(N) (64 = 8 x 8): every thread of a group has
// one DFT of each step, and a thread holds half the values of the 16 x 4
// split.
constexpr int kPkBz = 4;
template <int N> using PkZSplit = SplitSq<N>;
template <int N>
__device__ __forceinline__ void pk_z(const PkArgs &a, float2 *smem, const float2 *tw) {
  constexpr int B = kPkBz, MS = 3;
  constexpr int NG = PkZSplit<N>::R1 * B * MS;
  constexpr int GPC = kPkThreads / NG;
  static_assert(GPC >= 1, "a z tile needs at most one CTA of threads");
  const Geo &g = a.g;
  const int nkx = (g.Nh + B - 1) / B;
  const int ntile = nkx * g.N1;
  const int grp = threadIdx.x / NG, tid = threadIdx.x % NG;
  const bool ing = grp < GPC;
  float2 *buf = smem + (ing ? grp : 0) * MS * N * B;
  const long long zstride = (long long)g.N1 * g.Nhp;
  for (int base = blockIdx.x * GPC; base < ntile; base += gridDim.x * GPC) {
    const int t = base + grp;
    const bool act = ing && t < ntile;
    const int tt = act ? t : 0;
    const int kx0 = (tt % nkx) * B, y = tt / nkx;
    if (act) {
      for (int e = tid; e < g.m * N * (B / 2); e += NG) {
        const int s = e / (N * (B / 2)), r = e % (N * (B / 2));
        const int z = r / (B / 2), b2 = (r % (B / 2)) * 2;
        if (kx0 + b2 < g.Nhp)
          *reinterpret_cast<float4 *>(buf + s * N * B + z * B + b2) = *reinterpret_cast<const float4 *>(
              a.W + ((long long)s * g.N2 + z) * zstride + (long long)y * g.Nhp + kx0 + b2);
      }
    }
    __syncthreads();
    z_tile_g<float, MODE_J, N, B, MS, true, 1, PkZSplit<N>>(g, buf, tw, a.zp, kx0, y, tid, act);
    if (act) {
      for (int e = tid; e < g.m * N * (B / 2); e += NG) {
        const int s = e / (N * (B / 2)), r = e % (N * (B / 2));
        const int z = r / (B / 2), b2 = (r % (B / 2)) * 2;
        if (kx0 + b2 < g.Nhp)
          *reinterpret_cast<float4 *>(a.W + ((long long)s * g.N2 + z) * zstride + (long long)y * g.Nhp + kx0 + b2) =
              *reinterpret_cast<const float4 *>(buf + s * N * B + z * B + b2);
      }
    }
    __syncthreads();
  }
}

// Least squares of a k-step Arnoldi run, in place on the CTA's shared copy
// of H (column j at H[j * (k + 1) + i], i <= j + 1) by Givens rotations:
// y minimises |beta e1 - H y|; then y[0] += beta, so that sum y_j V_j = x +
// r0.  One thread; g, cs, sn are shared scratch of k + 1 entries.
__device__ __forceinline__ void pk_lsq(int k, double *H, double beta, double *y, double *gv, double *cs,
                                       double *sn) {
  const int ld = k + 1;
  for (int i = 0; i <= k; ++i) gv[i] = 0.0;
  gv[0] = beta;
  for (int j = 0; j < k; ++j) {
    double *col = H + j * ld;
    for (int i = 0; i < j; ++i) {
      const double p = col[i], q = col[i + 1];
      col[i] = cs[i] * p + sn[i] * q;
      col[i + 1] = -sn[i] * p + cs[i] * q;
    }
    const double p = col[j], q = col[j + 1];
    const double r = hypot(p, q);
    cs[j] = r == 0.0 ? 1.0 : p / r;
    sn[j] = r == 0.0 ? 0.0 : q / r;
    col[j] = r;
    gv[j + 1] = -sn[j] * gv[j];
    gv[j] = cs[j] * gv[j];
  }
  for (int i = k - 1; i >= 0; --i) {
    double s = gv[i];
    for (int l = i + 1; l < k; ++l) s -= H[l * ld + i] * y[l];
    y[i] = H[i * ld + i] != 0.0 ? s / H[i * ld + i] : 0.0;
  }
  if (k > 0) y[0] += beta;
}

// Shared memory of the phases (dynamic part): the three twiddle tables and
// the largest work tile (PLANE: a plane's row tile and its column tile).
template <int M, int N, bool PLANE = false> __host__ __device__ constexpr size_t pk_smem() {
  constexpr size_t xs = PLANE ? (size_t)N * (LayRow<M, PkSplit<M>::R2>::RS + pk_ncp<M>())
                              : (size_t)pk_rx<M>() * LayRow<M, PkSplit<M>::R2>::RS;
  constexpr size_t ys = PLANE ? 0 : (size_t)(kPkThreads / (Split<N>::R1 * 16)) * N * 16;
  constexpr size_t zs = (size_t)(kPkThreads / (PkZSplit<N>::R1 * kPkBz * 3)) * 3 * N * kPkBz;
  constexpr size_t tile = xs > ys ? (xs > zs ? xs : zs) : (ys > zs ? ys : zs);
  return sizeof(float2) * (M + 2 * N + tile);
}

// Grid barriers of one GMRES step: XF Y Z YI XI, or XY Z YXI with PLANE.
template <bool PLANE> __host__ __device__ constexpr int pk_phases() { return PLANE ? 3 : 5; }

// PLANE: every CTA owns whole (site, z) planes in the x phases, so that the
// y transforms ride in them (XY: update, c'_H, r2c along x, forward y; YXI:
// inverse y, c2r along x, dots) and a step has three grid barriers, not five.
template <int M, int N, bool PLANE = false>
__global__ void __launch_bounds__(kPkThreads, 2) k_coarse_gmres(PkArgs a) {
  constexpr int RXP = PLANE ? N : pk_rx<M>();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float2 *twx = reinterpret_cast<float2 *>(smem_raw);
  float2 *twy = twx + M;
  float2 *twz = twy + N;
  float2 *tile = twz + N;
  __shared__ double sH[kPkMaxSteps * (kPkMaxSteps + 1)];
  __shared__ double sS[kPkMaxSteps + 1];  // s_j = |V_j|
  __shared__ double sD[kVecMax];          // summed dot partials
  __shared__ float sC[kPkMaxSteps];       // update coefficients D_i / s_i^2
  __shared__ double sY[kPkMaxSteps];
  __shared__ float *sV[kPkMaxSteps + 1];  // the basis pointers, indexed at run time
  const int tid = threadIdx.x;
  const int k = a.k;
  if (tid <= kPkMaxSteps) sV[tid] = a.V[tid];
  if (a.trace && blockIdx.x == 0 && tid == 0) a.trace[0] = global_ns();
  for (int q = tid; q < M; q += kPkThreads) twx[q] = a.twx[q];
  for (int q = tid; q < N; q += kPkThreads) {
    twy[q] = a.twy[q];
    twz[q] = a.twz[q];
  }
  const float scale = 1.0f / (float)a.g.Nr;
  unsigned gen = 0;
  __syncthreads();  // sV and the twiddles are written before any thread reads them

  // P0: |r|^2
  {
    const long long nw = a.g.Nr * a.g.m / 4;
    double s2 = 0.0;
    for (long long i = (long long)blockIdx.x * kPkThreads + tid; i < nw; i += (long long)gridDim.x * kPkThreads) {
      const float4 v = reinterpret_cast<const float4 *>(sV[0])[i];
      s2 += (double)(v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w);
    }
    pk_block_sum(s2, a.pnrm);
  }
  if (!grid_sync(a.bar, ++gen, a.err, a.trace, a.trace_cta)) return;
  pk_sum_partials(a.pnrm, 1, gridDim.x, 1, sD);
  if (tid == 0) sS[0] = sqrt(fmax(sD[0], 0.0));
  __syncthreads();

  for (int j = 0; j <= k; ++j) {
    // the Gram-Schmidt update of V_j against V_0 .. V_{j-1} (coefficients
    // from the dot partials of the last XI phase), then its transform
    double nrm2 = 0.0;
    if (j > 0) {
      pk_sum_partials(a.pdot, kVecMax, gridDim.x, j, sD);
      if (tid < j) {
        const double si = sS[tid];
        sH[(j - 1) * (k + 1) + tid] = si > 0.0 ? sD[tid] / si : 0.0;  // h_{i,j-1} = <V_i/s_i, J V_{j-1}/s_{j-1}>
        sC[tid] = si > 0.0 ? (float)(sD[tid] / (si * si)) : 0.f;
      }
      __syncthreads();
    }
    pk_xf<M, RXP, PLANE, N>(a, sV, j, j, sC, j < k, tile, twx, twy, nrm2);
    if (j > 0) pk_block_sum(nrm2, a.pnrm + (j & 1) * gridDim.x);
    if (!grid_sync(a.bar, ++gen, a.err, a.trace, a.trace_cta)) return;
    if (j > 0) {
      pk_sum_partials(a.pnrm + (j & 1) * gridDim.x, 1, gridDim.x, 1, sD);
      if (tid == 0) {
        sS[j] = sqrt(fmax(sD[0], 0.0));
        sH[(j - 1) * (k + 1) + j] = sS[j];
      }
      __syncthreads();
    }
    if (j == k) break;
    if constexpr (!PLANE) {
      pk_y<N, false>(a, tile, twy);
      if (!grid_sync(a.bar, ++gen, a.err, a.trace, a.trace_cta)) return;
    }
    pk_z<N>(a, tile, twz);
    if (!grid_sync(a.bar, ++gen, a.err, a.trace, a.trace_cta)) return;
    if constexpr (!PLANE) {
      pk_y<N, true>(a, tile, twy);
      if (!grid_sync(a.bar, ++gen, a.err, a.trace, a.trace_cta)) return;
    }
    // V_{j+1} = J (V_j / s_j) = (X / N - V_j) / s_j
    const double sj = sS[j];
    const float inv = sj > 0.0 ? (float)(1.0 / sj) : 0.f;
    __shared__ double sdot[kPkMaxSteps][kPkThreads / 32];
    for (int q = tid; q < kPkMaxSteps * (kPkThreads / 32); q += kPkThreads) (&sdot[0][0])[q] = 0.0;
    __syncthreads();
    pk_xi<M, RXP, PLANE, N>(a, sV, j, scale * inv, inv, tile, twx, twy, sdot);
    if (tid <= j) {
      double t = 0.0;
      for (int w = 0; w < kPkThreads / 32; ++w) t += sdot[tid][w];
      a.pdot[(long long)blockIdx.x * kVecMax + tid] = t;
    }
    if (!grid_sync(a.bar, ++gen, a.err, a.trace, a.trace_cta)) return;
  }

  // least squares (every CTA, bitwise alike), then out = sum_j y_j V_j / s_j
  if (tid == 0) {
    __shared__ double sG[kPkMaxSteps + 1], sCs[kPkMaxSteps], sSn[kPkMaxSteps];
    if (blockIdx.x == 0)
      for (int q = 0; q < k * (k + 1); ++q) a.H[q] = sH[q];
    pk_lsq(k, sH, sS[0], sY, sG, sCs, sSn);
    if (blockIdx.x == 0) {
      a.aux[0] = sS[0];
      for (int i = 0; i < k; ++i) a.aux[1 + i] = sY[i];
    }
    for (int i = 0; i < k; ++i) sY[i] = sS[i] > 0.0 ? sY[i] / sS[i] : 0.0;
  }
  __syncthreads();
  const long long nw = a.g.Nr * a.g.m / 4;
  for (long long i = (long long)blockIdx.x * kPkThreads + tid; i < nw; i += (long long)gridDim.x * kPkThreads) {
    float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int q = 0; q < k; ++q) {
      const float c = (float)sY[q];
      const float4 v = reinterpret_cast<const float4 *>(sV[q])[i];
      o.x += c * v.x; o.y += c * v.y; o.z += c * v.z; o.w += c * v.w;
    }
    reinterpret_cast<float4 *>(a.out)[i] = o;
  }
  if (a.trace && blockIdx.x == 0 && tid == 0) a.trace[gen + 1] = global_ns();
}

}  // namespace rism
