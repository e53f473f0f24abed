// rism1d.cpp -- 1D RISM / DRISM pure-solvent solve producing the solvent
// susceptibility chi(k) = omega(k) + rho h(k) that the 3D solute solve
// consumes (rism_solvent / rism_vv, rism.f90:57-102, 310-583).
//
// CPU code: it runs once per solvent on m*m*nrad unknowns (36864 for
// 3-site water at nrad = 4096).  Radial Fourier transforms are DST-IV
// (FFTW RODFT11 in the reference, rism-dst.c:41-55, fft.f90:121-170),
// computed here through a complex FFT of length 2 nrad.  The non-linear
// solve is Newton-GMRES on r t(r) (rism.f90:415-437) with central-difference
// Jacobian products; only the fixed point matters.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "rism3d.h"

namespace {

using cplx = std::complex<double>;
const double kPi = 3.14159265358979323846;
const double kEps0Inv = 331.84164;  // units.f90:50
const double kAlpha = 1.2;          // units.f90:61

// ------------------------------------------------------------ complex FFT
// Stockham radix-4/2/3, out of place, unnormalised, sign = +1 or -1.
struct Fft {
  int n = 0;
  std::vector<int> rad;
  std::vector<cplx> tw;  // exp(sign 2 pi i q / n)
  std::vector<cplx> a, b;
  void init(int n_, int sign) {
    n = n_;
    rad.clear();
    int m = n;
    while (m % 4 == 0) { rad.push_back(4); m /= 4; }
    while (m % 2 == 0) { rad.push_back(2); m /= 2; }
    while (m % 3 == 0) { rad.push_back(3); m /= 3; }
    tw.resize(n);
    for (int q = 0; q < n; ++q) {
      const long double ang = sign * 2.0L * 3.141592653589793238462643383279502884L * q / n;
      tw[q] = cplx((double)cosl(ang), (double)sinl(ang));
    }
    a.resize(n);
    b.resize(n);
  }
  bool ok() const {
    int m = n;
    for (int r : rad) m /= r;
    return m == 1;
  }
  // in-place on a; a and b are the ping-pong buffers
  void run(int sign) {
    int Ns = 1;
    const cplx w3 = std::polar(1.0, sign * 2 * kPi / 3);
    for (int R : rad) {
      const int nR = n / R;
      const int tws = n / (Ns * R);
      for (int j = 0; j < nR; ++j) {
        const int k = j % Ns;
        cplx v[4];
        for (int r = 0; r < R; ++r) v[r] = a[j + r * nR] * (r && k ? tw[r * k * tws] : cplx(1, 0));
        cplx y[4];
        if (R == 2) {
          y[0] = v[0] + v[1];
          y[1] = v[0] - v[1];
        } else if (R == 4) {
          const cplx t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3];
          const cplx d = v[1] - v[3];
          const cplx t3 = sign > 0 ? cplx(-d.imag(), d.real()) : cplx(d.imag(), -d.real());
          y[0] = t0 + t2; y[2] = t0 - t2; y[1] = t1 + t3; y[3] = t1 - t3;
        } else {
          y[0] = v[0] + v[1] + v[2];
          y[1] = v[0] + w3 * v[1] + w3 * w3 * v[2];
          y[2] = v[0] + w3 * w3 * v[1] + w3 * v[2];
        }
        const int base = (j / Ns) * Ns * R + k;
        for (int r = 0; r < R; ++r) b[base + r * Ns] = y[r];
      }
      std::swap(a, b);
      Ns *= R;
    }
  }
};

// DST-IV of length n: y_k = 2 sum_j x_j sin(pi (2j+1)(2k+1) / (4n)), through
// one length-2n inverse-direction complex FFT with pre/post phases.
struct Dst4 {
  int n = 0;
  Fft fft;
  std::vector<cplx> pre, post;
  bool init(int n_) {
    n = n_;
    fft.init(2 * n, +1);
    if (!fft.ok()) return false;
    pre.resize(n);
    post.resize(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int j = 0; j < n; ++j) {
      const long double a = pi * j / (2.0L * n);
      pre[j] = cplx((double)cosl(a), (double)sinl(a));
      const long double b = pi * (2 * j + 1) / (4.0L * n);
      post[j] = cplx((double)cosl(b), (double)sinl(b));
    }
    return true;
  }
  void run(const double *x, double *y) {
    for (int j = 0; j < n; ++j) fft.a[j] = x[j] * pre[j];
    for (int j = n; j < 2 * n; ++j) fft.a[j] = 0.0;
    fft.run(+1);
    for (int k = 0; k < n; ++k) y[k] = 2.0 * (post[k] * fft.a[k]).imag();
  }
};

// ----------------------------------------------------------- small linalg
// Symmetric eigenproblem by cyclic Jacobi (n <= 3); columns of V.
void jacobi_eig(int n, double *A, double *e, double *V) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) V[i * n + j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[p * n + q] * A[p * n + q];
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) e[i] = A[i * n + i];
}

// Solve A X = B in place (A m x m, B m x m), partial pivoting.
void solve_mm(int m, double *A, double *B) {
  for (int c = 0; c < m; ++c) {
    int p = c;
    for (int r = c + 1; r < m; ++r)
      if (std::fabs(A[r * m + c]) > std::fabs(A[p * m + c])) p = r;
    if (p != c)
      for (int k = 0; k < m; ++k) { std::swap(A[c * m + k], A[p * m + k]); std::swap(B[c * m + k], B[p * m + k]); }
    for (int r = c + 1; r < m; ++r) {
      const double f = A[r * m + c] / A[c * m + c];
      for (int k = c; k < m; ++k) A[r * m + k] -= f * A[c * m + k];
      for (int k = 0; k < m; ++k) B[r * m + k] -= f * B[c * m + k];
    }
  }
  for (int c = m - 1; c >= 0; --c)
    for (int k = 0; k < m; ++k) {
      double s = B[c * m + k];
      for (int j = c + 1; j < m; ++j) s -= A[c * m + j] * B[j * m + k];
      B[c * m + k] = s / A[c * m + c];
    }
}

// ------------------------------------------------------------ physics
double j0s(double x) {  // bessel.f90:36-58
  if (std::fabs(x) < 0.5) {
    const double y = x * x;
    return 1 + y * (-1 / 6.0 + y * (1 / 120.0 + y * (-1 / 5040.0 + y * (1 / 362880.0 + y * (-1 / 39916800.0 +
                    y * (1 / 6227020800.0))))));
  }
  return std::sin(x) / x;
}
double j1s(double x) {  // bessel.f90:61-91
  if (std::fabs(x) < 0.25) {
    const double y = x * x;
    return x / 3 * (1 + y * (-1 / 10.0 + y * (1 / 280.0 + y * (-1 / 15120.0 + y * (1 / 1330560.0 +
                    y * (-1 / 172972800.0))))));
  }
  return (std::sin(x) / x - std::cos(x)) / x;
}

double closure_c(int method, double bv, double t) {  // closures.f90:107-128
  const double x = -bv + t;
  if (method == RISM3D_HNC) return std::expm1(x) - t;
  if (method == RISM3D_KH) return x <= 0 ? std::expm1(x) - t : -bv;
  if (method == RISM3D_PY) return std::exp(-bv) * (1 + t) - 1 - t;
  const int n = method - RISM3D_PSE0;
  if (x < 0) return std::expm1(x) - t;
  double c = 1, y = 0;
  for (int k = n; k >= 1; --k) { y = x * y + c; c *= k; }
  return (x / c) * y - t;
}

double form(int method, double x, double h, double c, double cl) {  // closures.f90:574-612
  const double base = -c - h * (c + cl) / 2;
  if (method == RISM3D_HNC) return base + h * h / 2;
  if (method == RISM3D_KH) return h < 0 ? base + h * h / 2 : base;
  if (method == RISM3D_PY) return base;
  if (h < 0) return base + h * h / 2;
  const int mm = method - RISM3D_PSE0 + 1;
  double f = 1, xm = 1;
  for (int k = 1; k <= mm; ++k) { f *= k; xm *= x; }
  return base + (h * h / 2 - xm / f);
}

struct Vv {
  int m, n, method;
  double beta, rho, eps, dr, dk;
  std::vector<double> r, k, vr, vk, wk, xk, wx;  // pair arrays [i][j][p]
  Dst4 dst;
  std::vector<double> buf, out;

  size_t at(int i, int j) const { return ((size_t)i * m + j) * n; }

  // fourier_rows (fft.f90:121-170) of every pair row, times scale
  void fourier(std::vector<double> &f, double scale) {
    for (int ij = 0; ij < m * m; ++ij) {
      double *row = f.data() + (size_t)ij * n;
      for (int p = 0; p < n; ++p) buf[p] = row[p] * (2.0 * n * (2 * p + 1));
      dst.run(buf.data(), out.data());
      for (int p = 0; p < n; ++p) row[p] = out[p] * (1.0 / (2 * p + 1)) * scale;
    }
  }

  // iterate_t (rism.f90:469-536) on r t(r)
  void residual(const std::vector<double> &rt, std::vector<double> &drt) {
    const size_t N = (size_t)m * m * n;
    std::vector<double> t(N), c(N);
    for (int ij = 0; ij < m * m; ++ij)
      for (int p = 0; p < n; ++p) t[(size_t)ij * n + p] = rt[(size_t)ij * n + p] / r[p];
    for (size_t q = 0; q < N; ++q) c[q] = closure_c(method, beta * vr[q], t[q]);
    fourier(c, dr * dr * dr);
    for (size_t q = 0; q < N; ++q) c[q] -= beta * vk[q];
    std::vector<double> dt(N);
    std::vector<double> C(m * m), W(m * m), H(m * m), T(m * m);
    for (int p = 0; p < n; ++p) {
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
          C[i * m + j] = c[at(i, j) + p];
          W[i * m + j] = wx[at(i, j) + p];
        }
      if (m == 1) {  // rism.f90:2458-2473
        const double cc = C[0];
        dt[p] = rho * (cc * cc) / (1 - rho * cc);
      } else {       // rism.f90:2476-2560
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) {
            double s = 0;
            for (int l = 0; l < m; ++l) s += W[i * m + l] * C[l * m + j];
            H[i * m + j] = s;
          }
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) T[i * m + j] = (i == j ? 1.0 : 0.0) - H[i * m + j] * rho;
        std::vector<double> HW(m * m);
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) {
            double s = 0;
            for (int l = 0; l < m; ++l) s += H[i * m + l] * W[l * m + j];
            HW[i * m + j] = s;
          }
        solve_mm(m, T.data(), HW.data());
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) dt[at(i, j) + p] = HW[i * m + j] - C[i * m + j];
      }
      if (eps != 0.0)
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) dt[at(i, j) + p] += xk[at(i, j) + p];
    }
    for (size_t q = 0; q < N; ++q) dt[q] -= beta * vk[q];
    fourier(dt, dk * dk * dk / std::pow(2 * kPi, 3));
    drt.resize(N);
    for (int ij = 0; ij < m * m; ++ij)
      for (int p = 0; p < n; ++p) {
        const size_t q = (size_t)ij * n + p;
        drt[q] = r[p] * (dt[q] - t[q]);
      }
  }
};

double norm2(const std::vector<double> &a) {
  double s = 0;
  for (double v : a) s += v * v;
  return std::sqrt(s);
}
double norminf(const std::vector<double> &a) {
  double s = 0;
  for (double v : a) s = std::max(s, std::fabs(v));
  return s;
}

// Newton-GMRES with central-difference J v and backtracking; returns iterations or -1.
template <typename F>
int newton_fd(F &&fun, std::vector<double> &x, double tol, int max_iter) {
  const size_t N = x.size();
  std::vector<double> f, ft, xt;
  fun(x, f);
  const int restart = 40;
  for (int it = 0; it < max_iter; ++it) {
    if (!(norminf(f) == norminf(f))) return -2;
    if (norminf(f) < tol) return it;
    // GMRES for J d = -f
    std::vector<std::vector<double>> V;
    std::vector<double> H((restart + 1) * restart, 0.0), cs(restart), sn(restart), g(restart + 1, 0.0);
    std::vector<double> d(N, 0.0);
    const double beta = norm2(f);
    V.push_back(std::vector<double>(N));
    for (size_t q = 0; q < N; ++q) V[0][q] = -f[q] / beta;
    g[0] = beta;
    const double xn = std::max(1.0, norm2(x));
    int kdim = 0;
    for (int j = 0; j < restart; ++j) {
      const double h = 1e-7 * xn;
      std::vector<double> xp(x), xm(x), fp, fm;
      for (size_t q = 0; q < N; ++q) { xp[q] += h * V[j][q]; xm[q] -= h * V[j][q]; }
      fun(xp, fp);
      fun(xm, fm);
      std::vector<double> w(N);
      for (size_t q = 0; q < N; ++q) w[q] = (fp[q] - fm[q]) / (2 * h);
      for (int i = 0; i <= j; ++i) {  // modified Gram-Schmidt
        double s = 0;
        for (size_t q = 0; q < N; ++q) s += w[q] * V[i][q];
        H[i * restart + j] = s;
        for (size_t q = 0; q < N; ++q) w[q] -= s * V[i][q];
      }
      const double hn = norm2(w);
      H[(j + 1) * restart + j] = hn;
      for (int i = 0; i < j; ++i) {
        const double a = H[i * restart + j], b = H[(i + 1) * restart + j];
        H[i * restart + j] = cs[i] * a + sn[i] * b;
        H[(i + 1) * restart + j] = -sn[i] * a + cs[i] * b;
      }
      const double a = H[j * restart + j], b = H[(j + 1) * restart + j];
      const double rr = std::hypot(a, b);
      cs[j] = rr == 0 ? 1 : a / rr;
      sn[j] = rr == 0 ? 0 : b / rr;
      H[j * restart + j] = rr;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      kdim = j + 1;
      if (hn == 0 || std::fabs(g[j + 1]) < 1e-4 * beta) break;
      V.push_back(std::vector<double>(N));
      for (size_t q = 0; q < N; ++q) V[j + 1][q] = w[q] / hn;
    }
    std::vector<double> y(kdim);
    for (int i = kdim - 1; i >= 0; --i) {
      double s = g[i];
      for (int l = i + 1; l < kdim; ++l) s -= H[i * restart + l] * y[l];
      y[i] = s / H[i * restart + i];
    }
    for (int i = 0; i < kdim; ++i)
      for (size_t q = 0; q < N; ++q) d[q] += y[i] * V[i][q];
    const double f0 = beta * beta;
    double lam = 1.0;
    bool ok = false;
    for (int ls = 0; ls < 30; ++ls) {
      xt = x;
      for (size_t q = 0; q < N; ++q) xt[q] += lam * d[q];
      fun(xt, ft);
      const double f1 = norm2(ft) * norm2(ft);
      if (f1 <= (1 - 2e-4 * lam) * f0) { ok = true; break; }
      lam *= 0.5;
    }
    if (!ok) return norminf(ft) < tol ? it : -1;
    x.swap(xt);
    f.swap(ft);
  }
  return norminf(f) < tol ? max_iter : -1;
}

}  // namespace

extern "C" int rism1d_solvent_chi(const rism3d_problem *pd, double dielectric, int m, const rism3d_site *sv,
                                  double *chi_out, double *t_out, double *mu_out) {
  if (!pd || !sv || !chi_out || m < 1 || m > 16 || pd->nrad < 4 || !(pd->rmax > 0)) return RISM3D_ERR_ARG;
  if (pd->closure < 0 || pd->closure > RISM3D_PSE7) return RISM3D_ERR_ARG;
  Vv P;
  P.m = m;
  P.n = pd->nrad;
  P.method = pd->closure;
  P.beta = pd->beta;
  P.rho = pd->rho;
  P.eps = dielectric;
  const int n = P.n;
  if (!P.dst.init(n)) return RISM3D_ERR_ARG;  // nrad must be 2^a 3^b
  P.buf.resize(n);
  P.out.resize(n);
  P.dr = pd->rmax / n;  // mkgrid, fft.f90:101-118
  P.dk = kPi / pd->rmax;
  P.r.resize(n);
  P.k.resize(n);
  for (int i = 0; i < n; ++i) {
    P.r[i] = (2 * (i + 1) - 1) * P.dr / 2;
    P.k[i] = (2 * (i + 1) - 1) * P.dk / 2;
  }
  const size_t N = (size_t)m * m * n;
  P.vr.assign(N, 0.0);
  P.vk.assign(N, 0.0);
  P.wk.assign(N, 0.0);
  P.xk.assign(N, 0.0);
  // force_field (rism.f90:2082-2162), Lorentz-Berthelot (1323-1350)
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      const double qab = sv[i].charge * sv[j].charge;
      const double sigma = (sv[i].sigma + sv[j].sigma) / 2;
      const double epsilon = std::sqrt(sv[i].epsilon * sv[j].epsilon);
      const double rab = std::sqrt(std::pow(sv[i].x[0] - sv[j].x[0], 2) + std::pow(sv[i].x[1] - sv[j].x[1], 2) +
                                   std::pow(sv[i].x[2] - sv[j].x[2], 2));
      for (int p = 0; p < n; ++p) {
        const double rr = P.r[p], kk = P.k[p];
        double v = kEps0Inv * qab * (std::erfc(kAlpha * rr) / rr);
        if (sigma != 0.0) {
          const double sr6 = 1 / std::pow(rr / sigma, 6);
          v += epsilon * (4 * sr6 * (sr6 - 1));
        }
        P.vr[P.at(i, j) + p] = v;
        P.vk[P.at(i, j) + p] = kEps0Inv * qab * (4 * kPi * std::exp(-kk * kk / (4 * kAlpha * kAlpha)) / (kk * kk));
        P.wk[P.at(i, j) + p] = j0s(kk * rab);  // omega_fourier, rism.f90:1994-2032
      }
    }
  if (dielectric != 0.0) {
    // dipole_correction (drism.f90:373-474) with local axes of dipole_axes
    double dip[3] = {0, 0, 0}, cen[3] = {0, 0, 0}, wsum = 0;
    for (int s = 0; s < m; ++s) {
      const double w = std::pow(sv[s].sigma, 3);
      wsum += w;
      for (int d = 0; d < 3; ++d) { dip[d] += sv[s].charge * sv[s].x[d]; cen[d] += w * sv[s].x[d]; }
    }
    for (int d = 0; d < 3; ++d) cen[d] /= wsum;
    const double mu2 = dip[0] * dip[0] + dip[1] * dip[1] + dip[2] * dip[2];
    const double dn = std::sqrt(mu2);
    if (!(dn > 1e-7)) return RISM3D_ERR_ARG;  // zero dipole: DRISM undefined
    const double ez[3] = {dip[0] / dn, dip[1] / dn, dip[2] / dn};
    // an orthonormal basis (e1, e2) of the plane normal to the dipole ...
    double e1[3];
    {
      const double ax[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      int best = 0;
      double bmin = 2;
      for (int a = 0; a < 3; ++a) {
        const double d = std::fabs(ax[a][0] * ez[0] + ax[a][1] * ez[1] + ax[a][2] * ez[2]);
        if (d < bmin) { bmin = d; best = a; }
      }
      const double dd = ax[best][0] * ez[0] + ax[best][1] * ez[1] + ax[best][2] * ez[2];
      double nn = 0;
      for (int d = 0; d < 3; ++d) { e1[d] = ax[best][d] - dd * ez[d]; nn += e1[d] * e1[d]; }
      nn = std::sqrt(nn);
      for (int d = 0; d < 3; ++d) e1[d] /= nn;
    }
    const double e2[3] = {ez[1] * e1[2] - ez[2] * e1[1], ez[2] * e1[0] - ez[0] * e1[2], ez[0] * e1[1] - ez[1] * e1[0]};
    // ... rotated onto the eigenvectors of the in-plane shape tensor
    double T2[4] = {0, 0, 0, 0};
    std::vector<double> d1(m), d2(m), d3(m);
    for (int s = 0; s < m; ++s) {
      const double w = std::pow(sv[s].sigma, 3) / wsum;
      double rel[3];
      for (int d = 0; d < 3; ++d) rel[d] = sv[s].x[d] - cen[d];
      const double a = rel[0] * e1[0] + rel[1] * e1[1] + rel[2] * e1[2];
      const double b = rel[0] * e2[0] + rel[1] * e2[1] + rel[2] * e2[2];
      d1[s] = a;
      d2[s] = b;
      d3[s] = rel[0] * ez[0] + rel[1] * ez[1] + rel[2] * ez[2];
      T2[0] += w * a * a; T2[1] += w * a * b; T2[2] += w * b * a; T2[3] += w * b * b;
    }
    double ev[2], V2[4];
    jacobi_eig(2, T2, ev, V2);
    std::vector<double> xl(m), yl(m);
    for (int s = 0; s < m; ++s) {
      xl[s] = d1[s] * V2[0] + d2[s] * V2[2];
      yl[s] = d1[s] * V2[1] + d2[s] * V2[3];
    }
    const double y = 4 * kPi * P.beta * kEps0Inv * P.rho * mu2 / 9;  // drism.f90:20-41
    const double sdip = 0.5;
    for (int p = 0; p < n; ++p) {
      const double kk = P.k[p];
      const double h = (dielectric - (1 + 3 * y)) / (P.rho * y) * std::exp(-(kk * sdip) * (kk * sdip) / 4);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
          const double fi = j0s(kk * xl[i]) * j0s(kk * yl[i]) * j1s(kk * d3[i]);
          const double fj = j0s(kk * xl[j]) * j0s(kk * yl[j]) * j1s(kk * d3[j]);
          P.xk[P.at(i, j) + p] = fi * h * fj;
        }
    }
  }
  P.wx.resize(N);
  for (size_t q = 0; q < N; ++q) P.wx[q] = P.wk[q] + (dielectric != 0.0 ? P.rho * P.xk[q] : 0.0);

  std::vector<double> rt(N, 0.0);
  if (t_out)  // optional initial guess t(r)
    for (int ij = 0; ij < m * m; ++ij)
      for (int p = 0; p < n; ++p) rt[(size_t)ij * n + p] = P.r[p] * t_out[(size_t)ij * n + p];
  const double tol = pd->norm_tol > 0 ? pd->norm_tol : 1e-12;
  const int it = newton_fd([&](const std::vector<double> &x, std::vector<double> &f) { P.residual(x, f); }, rt,
                           tol, pd->max_iter > 0 ? pd->max_iter : 200);
  if (it == -2) return RISM3D_ERR_NAN;
  if (it < 0) return RISM3D_ERR_NOT_CONVERGED;
  // chi = omega + rho h, h(k) = FT(c + t) (rism.f90:445-453)
  std::vector<double> t(N), h(N);
  for (int ij = 0; ij < m * m; ++ij)
    for (int p = 0; p < n; ++p) t[(size_t)ij * n + p] = rt[(size_t)ij * n + p] / P.r[p];
  for (size_t q = 0; q < N; ++q) h[q] = closure_c(P.method, P.beta * P.vr[q], t[q]) + t[q];
  P.fourier(h, P.dr * P.dr * P.dr);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j)
      for (int p = 0; p < n; ++p)  // C layout [m][m][nrad] (rism.f90:2749-2761)
        chi_out[P.at(j, i) + p] = P.wk[P.at(i, j) + p] + P.rho * h[P.at(i, j) + p];
  if (t_out) std::memcpy(t_out, t.data(), sizeof(double) * N);
  if (mu_out) {  // chempot (closures.f90 chempot) with integrate (fft.f90)
    double acc = 0;
    for (int p = n - 1; p >= 0; --p) {
      double dens = 0;
      for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) {
          const size_t q = P.at(i, j) + p;
          const double c = closure_c(P.method, P.beta * P.vr[q], t[q]);
          const double rr = P.r[p];
          const double vl = sv[i].charge * sv[j].charge * kEps0Inv * (std::erf(kAlpha * rr) / rr);
          dens += form(P.method, -P.beta * P.vr[q] + t[q], c + t[q], c, -P.beta * vl);
        }
      acc += dens * std::pow(2 * (p + 1) - 1, 2) / 4;
    }
    *mu_out = 4 * kPi * acc * (P.rho * std::pow(P.dr, 3) / P.beta);
  }
  return RISM3D_OK;
}
