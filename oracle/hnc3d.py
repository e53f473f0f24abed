"""3D-RISM solute solve -- restatement of hnc3d_solute_solve (hnc3d.c:1762-2350).

Test infrastructure only (see oracle/__init__.py).

Layout: real fields are NumPy arrays [N2][N1][N0] (N0 = x fastest, the
DMDA order of bgy3d-fftw3.c:295-339); k-fields are [N2][N1][N0/2+1]
(FFTW r2c halving the stride-1 dimension, bgy3d-fftw3.c:374-385).
FFTW's unnormalised r2c/c2r map onto scipy.fft rfftn / (N * irfftn).
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft
import scipy.special
import scipy.sparse.linalg as sla

from . import closures as cl
from . import newton
from .rism1d import EPSILON0INV, coulomb_long_fourier, mkgrid

G = 1.2                          # G_COULOMB_INVERSE_RANGE, bgy3d-solvents.h:9
RMIN = 0.2                       # bgy3d-solutes.c:68, 220
_WORKERS = 8


# ------------------------------------------------------- pair primitives
def lj0(r):
    """bgy3d-solutes.c:46-53."""
    p6 = np.power(r, -6.0)
    return 4 * p6 * (p6 - 1)


def lj1(r):
    """bgy3d-solutes.c:56-62."""
    p6 = np.power(r, -6.0)
    return 4 * p6 * (6 - 12 * p6) / r


def ljcap0(r):
    """bgy3d-solutes.c:101-114: parabola cap below RMIN."""
    R = RMIN
    b = lj1(R) / (2 * R)
    a = lj0(R)
    rs = np.where(r >= R, r, 1.0)
    return np.where(r >= R, lj0(rs), a + b * (r - R) * (r + R))


def ljcap1(r):
    """bgy3d-solutes.c:118-129."""
    R = RMIN
    b = lj1(R) / (2 * R)
    rs = np.where(r >= R, r, 1.0)
    return np.where(r >= R, lj1(rs), 2 * b * r)


def cl0(r):
    """bgy3d-solutes.c:147-159: erf(r)/r with Taylor branch below 0.02."""
    r = np.asarray(r, dtype=np.float64)
    r2 = r ** 2
    taylor = (2 / np.sqrt(np.pi)) * (1. + r2 * (-1. / 3. + r2 * (1. / 10. + r2 * (-1. / 42.))))
    rs = np.where(r >= 0.02, r, 1.0)
    return np.where(r >= 0.02, scipy.special.erf(rs) / rs, taylor)


def cl1(r):
    """bgy3d-solutes.c:181-193."""
    r = np.asarray(r, dtype=np.float64)
    r2 = r ** 2
    rs = np.where(r >= 0.02, r, 1.0)
    big = ((2 / np.sqrt(np.pi)) * rs * np.exp(-rs ** 2) - scipy.special.erf(rs)) / rs ** 2
    taylor = -(4 / (3 * np.sqrt(np.pi))) * r * (1. + r2 * (-3. / 5. + r2 * (3. / 14. + r2 * (-1. / 18.))))
    return np.where(r >= 0.02, big, taylor)


def cs0(r):
    """bgy3d-solutes.c:197-201."""
    return scipy.special.erfc(r) / r


def cs1(r):
    """bgy3d-solutes.c:205-210."""
    r2 = r ** 2
    return -(scipy.special.erfc(r) + (2 / np.sqrt(np.pi)) * r * np.exp(-r2)) / r2


def cscap0(r):
    """bgy3d-solutes.c:230-243."""
    R = RMIN
    b = cs1(R) / (2 * R)
    a = cs0(R)
    rs = np.where(r >= R, r, 1.0)
    return np.where(r >= R, cs0(rs), a + b * (r - R) * (r + R))


def cscap1(r):
    """bgy3d-solutes.c:245-257."""
    R = RMIN
    b = cs1(R) / (2 * R)
    rs = np.where(r >= R, r, 1.0)
    return np.where(r >= R, cs1(rs), 2 * b * r)


def ccap1(r):
    """bgy3d-solutes.c:275-283: capped full Coulomb derivative."""
    R = RMIN
    rs = np.where(r >= R, r, 1.0)
    return np.where(r >= R, -1.0 / (rs * rs), cscap1(r) + cl1(r))


# ------------------------------------------------------------- grids
def kfreq(i, n):
    """bgy3d.h:162."""
    return np.where(i <= n // 2, i, i - n)


def rgrid(N, L, zs=slice(None)):
    """vec_rmap3 (bgy3d-vec.h:578-607): r = i h - L/2, arrays [z][y][x]
    (the z planes ``zs`` only)."""
    h = [L[d] / N[d] for d in range(3)]
    ax = [np.arange(N[d]) * h[d] - L[d] / 2 for d in range(3)]
    return ax[0][None, None, :], ax[1][None, :, None], ax[2][zs][:, None, None]


def kgrid(N, L, zs=slice(None)):
    """vec_kmap3 (bgy3d-vec.h:613-648): k = KFREQ(i) * 2 pi / L on [N2][N1][N0/2+1]
    (the kz planes ``zs`` only)."""
    dk = [2 * np.pi / L[d] for d in range(3)]
    i0 = np.arange(N[0] // 2 + 1)
    i1 = np.arange(N[1])
    i2 = np.arange(N[2])[zs]
    k0 = (kfreq(i0, N[0]) * dk[0])[None, None, :]
    k1 = (kfreq(i1, N[1]) * dk[1])[None, :, None]
    k2 = (kfreq(i2, N[2]) * dk[2])[:, None, None]
    sign = ((-1.0) ** kfreq(i0, N[0]))[None, None, :] * \
           ((-1.0) ** kfreq(i1, N[1]))[None, :, None] * \
           ((-1.0) ** kfreq(i2, N[2]))[:, None, None]
    return k0, k1, k2, sign


def kabs(N, L, zs=slice(None)):
    k0, k1, k2, _ = kgrid(N, L, zs)
    return np.sqrt((k0 ** 2 + k1 ** 2) + k2 ** 2)


def interp(x, xtab, dx):
    """bgy3d-vec.c:22-46: nearest entry plus a (mostly central) slope."""
    n = xtab.size
    ix = x / dx - 0.5
    i = (ix + 0.5).astype(np.int64)
    if np.any(i < 0) or np.any(i >= n):
        raise ValueError("interp: |k| outside the radial table")
    ip = np.where(i < n - 2, i + 1, i)
    im = np.where(i > 1, i - 1, i)
    fi = (xtab[ip] - xtab[im]) / (ip - im)
    return xtab[i] + fi * (ix - i)


# ------------------------------------------------------------- setup
def solute_field(N, L, solvent, solute, zs=slice(None)):
    """field0 (bgy3d-solutes.c:343-377): v[m][N2][N1][N0] (z planes ``zs``)."""
    x, y, z = rgrid(N, L, zs)
    m = len(solvent)
    v = np.zeros((m, z.shape[0], N[1], N[0]))
    for i, a in enumerate(solvent):
        e = np.zeros((z.shape[0], N[1], N[0]))
        for b in solute:
            eab = np.sqrt(a["epsilon"] * b["epsilon"])
            sab = 0.5 * (a["sigma"] + b["sigma"])
            qab = a["charge"] * b["charge"] * EPSILON0INV
            bx = b["x"]
            rab = np.sqrt((x - bx[0]) ** 2 + (y - bx[1]) ** 2 + (z - bx[2]) ** 2)
            e = e + (eab * ljcap0(rab / sab) + qab * G * cscap0(G * rab))
        v[i] = e
    return v


def solute_field1(N, L, solvent, solute, u, dim):
    """field1 (bgy3d-solutes.c:381-468) for a unit displacement of site u along dim."""
    x, y, z = rgrid(N, L)
    b = solute[u]
    ab = [x - b["x"][0], y - b["x"][1], z - b["x"][2]]
    rab = np.sqrt(ab[0] ** 2 + ab[1] ** 2 + ab[2] ** 2)
    drab = np.where(rab > 0.0, -ab[dim] / np.where(rab > 0.0, rab, 1.0), 0.0)
    out = np.zeros((len(solvent), N[2], N[1], N[0]))
    for i, a in enumerate(solvent):
        eab = np.sqrt(a["epsilon"] * b["epsilon"])
        sab = 0.5 * (a["sigma"] + b["sigma"])
        qab = a["charge"] * b["charge"] * EPSILON0INV
        out[i] = drab * ((eab / sab) * ljcap1(rab / sab) + qab * G * G * ccap1(G * rab))
    return out


def coulomb_long(N, L, solute):
    """bgy3d-solutes.c:795-815: uc(r) = (1/eps0) sum q G cl0(G r)."""
    x, y, z = rgrid(N, L)
    s = np.zeros((N[2], N[1], N[0]))
    for b in solute:
        bx = b["x"]
        r = np.sqrt((x - bx[0]) ** 2 + (y - bx[1]) ** 2 + (z - bx[2]) ** 2)
        s = s + b["charge"] * G * cl0(G * r)
    return EPSILON0INV * s


def form_factor_centered(N, L, solute, zs=slice(None)):
    """solute_form (bgy3d-solutes.c:633-660): sum q e^{-ik.x} times (-1)^(ix+iy+iz)
    (kz planes ``zs``)."""
    k0, k1, k2, sign = kgrid(N, L, zs)
    f = np.zeros((k2.shape[0], N[1], N[0] // 2 + 1), dtype=np.complex128)
    for b in solute:
        bx = b["x"]
        f = f + b["charge"] * np.exp(-1j * ((k0 * bx[0] + k1 * bx[1]) + k2 * bx[2]))
    return f * sign


def renorm_kernel(solvent, chi, rmax, alpha=G):
    """rism_solvent_renorm (rism.f90:141-208): s_i(k) = sum_j chi_ij q_j 4 pi e^{-k^2/4a^2}/k^2."""
    nrad = chi.shape[-1]
    _, _, k, _ = mkgrid(rmax, nrad)
    v = coulomb_long_fourier(k, alpha)
    q = np.array([s["charge"] for s in solvent])
    m = len(solvent)
    s = np.zeros((m, nrad))
    for i in range(m):
        x = np.zeros(nrad)
        for j in range(m):
            x = x + chi[j, i] * q[j]
        s[i] = x * v
    return s


class Problem:
    """Everything hnc3d_solute_solve sets up before SNES (hnc3d.c:1790-1966).

    ``threads`` > 1 evaluates the pointwise work (setup, closure, OZ
    contraction, scaling) on z-slabs in a thread pool and the FFTs with
    that many workers: the same arithmetic per grid point, for timing the
    restatement on every host core."""

    def __init__(self, N, L, beta, rho, closure, solvent, solute, chi, rmax, renorm=True, chi3=None, threads=1):
        """chi: [m][m][nrad] radial chi table, or None with chi3 = chi - 1 on
        the k grid (packed pairs [m(m+1)/2][N2][N1][N0/2+1], complex), the
        --solvent-3d kernel read from x%d%d-fft.bin (solvent_kernel_file,
        hnc3d.c:1432-1437), which implies the no-renorm form (1575-1587)."""
        self.N = tuple(int(n) for n in N)
        self.L = tuple(float(l) for l in L)
        self.h = tuple(self.L[d] / self.N[d] for d in range(3))
        self.beta, self.rho, self.closure = float(beta), float(rho), int(closure)
        self.solvent, self.solute = solvent, solute
        self.m = len(solvent)
        self.renorm = renorm
        self.h3 = self.h[0] * self.h[1] * self.h[2]
        self.L3 = self.L[0] * self.L[1] * self.L[2]
        self.threads = max(1, int(threads))
        self.workers = self.threads if self.threads > 1 else _WORKERS
        self._pool = ThreadPoolExecutor(self.threads) if self.threads > 1 else None
        m = self.m
        nk = (self.N[2], self.N[1], self.N[0] // 2 + 1)
        if chi3 is not None:
            renorm = self.renorm = False
            self.chi_fft = np.zeros((m, m) + nk, dtype=complex)
            p = 0
            for i in range(m):
                for j in range(i + 1):
                    self.chi_fft[i, j] = self.chi_fft[j, i] = chi3[p]
                    p += 1
        else:
            dk = np.pi / rmax
            self.chi_fft = np.zeros((m, m) + nk)
        self.charge = np.array([s["charge"] for s in solvent])
        if renorm:
            srad = renorm_kernel(solvent, chi, rmax)
            self.tau_fft = np.zeros((m,) + nk, dtype=complex)
            self.v_long_fft = None
        else:
            self.tau_fft = None
            self.v_long_fft = np.zeros(nk, dtype=complex)
        self.v = np.zeros((m, self.N[2], self.N[1], self.N[0]))

        def setup(a, b):
            zs = slice(a, b)
            kk = kabs(self.N, self.L, zs)
            if chi3 is None:
                for i in range(m):
                    for j in range(i + 1):
                        tab = chi[i, j] - (1.0 if i == j else 0.0)
                        self.chi_fft[i, j, a:b] = interp(kk, tab, dk)
                        self.chi_fft[j, i, a:b] = self.chi_fft[i, j, a:b]
            F = form_factor_centered(self.N, self.L, solute, zs)
            if renorm:
                for i in range(m):
                    self.tau_fft[i, a:b] = interp(kk, srad[i], dk) * F
            else:
                # bgy3d-force.h:139-148 coulomb_long_fourier(k, q2=1, G), corner;
                # centred through F (bgy3d-solutes.c:766-792)
                self.v_long_fft[a:b] = EPSILON0INV * coulomb_long_fourier(kk, G) * F
            self.v[:, a:b] = solute_field(self.N, self.L, solvent, solute, zs)

        self._each_slab(setup)

    def _each_slab(self, fn):
        """fn(a, b) over z-slabs [a, b) of the grid (k grids: kz planes)."""
        n2 = self.N[2]
        if self._pool is None:
            fn(0, n2)
            return
        k = min(n2, 4 * self.threads)
        cuts = [n2 * q // k for q in range(k + 1)]
        for f in [self._pool.submit(fn, cuts[q], cuts[q + 1]) for q in range(k) if cuts[q] < cuts[q + 1]]:
            f.result()

    # -- FFT MatShell (bgy3d-fftw3.c:229-265), unnormalised ------------
    def fft(self, x):
        return scipy.fft.rfftn(x, axes=(-3, -2, -1), workers=self.workers)

    def ifft(self, y):
        n = self.N[0] * self.N[1] * self.N[2]
        return scipy.fft.irfftn(y, s=(self.N[2], self.N[1], self.N[0]), axes=(-3, -2, -1),
                                workers=self.workers) * n

    def star(self, c_fft):
        """hnc3d.c:1114-1138."""
        return np.einsum("ijk...,jk...->ik...", self.chi_fft.reshape(self.m, self.m, -1),
                         c_fft.reshape(self.m, -1)).reshape(c_fft.shape)

    def _star_slab(self, cf, a, b):
        """star on the kz planes [a, b): t_i = sum_j (chi-1)_ij c_j."""
        out = np.zeros_like(cf)
        for i in range(self.m):
            for j in range(self.m):
                out[i] += self.chi_fft[i, j, a:b] * cf[j]
        return out

    def iterate_t1(self, T):
        """hnc3d.c:1183-1285: dT = (chi-1)*c(t) [- beta/eps0 tau] - t."""
        beta = self.beta
        if self._pool is not None:
            return self._iterate_t1_slabs(T)
        c = cl.closure(self.closure, beta, self.v, T)
        c_fft = self.fft(c) * self.h3
        if not self.renorm:
            c_fft = c_fft - (beta * self.charge)[:, None, None, None] * self.v_long_fft
        t_fft = self.star(c_fft)
        if self.renorm:
            t_fft = t_fft - (beta * EPSILON0INV) * self.tau_fft
        else:
            t_fft = t_fft - (beta * self.charge)[:, None, None, None] * self.v_long_fft
        return self.ifft(t_fft) * (1.0 / self.L3) - T

    def _iterate_t1_slabs(self, T):
        beta = self.beta
        c = np.empty_like(T)

        def clo(a, b):
            c[:, a:b] = cl.closure(self.closure, beta, self.v[:, a:b], T[:, a:b])

        self._each_slab(clo)
        c_fft = self.fft(c)
        t_fft = np.empty_like(c_fft)

        def oz(a, b):
            cf = c_fft[:, a:b] * self.h3
            if not self.renorm:
                cf = cf - (beta * self.charge)[:, None, None, None] * self.v_long_fft[a:b]
            tf = self._star_slab(cf, a, b)
            if self.renorm:
                tf -= (beta * EPSILON0INV) * self.tau_fft[:, a:b]
            else:
                tf -= (beta * self.charge)[:, None, None, None] * self.v_long_fft[a:b]
            t_fft[:, a:b] = tf

        self._each_slab(oz)
        r = self.ifft(t_fft)

        def fin(a, b):
            r[:, a:b] *= 1.0 / self.L3
            r[:, a:b] -= T[:, a:b]

        self._each_slab(fin)
        return r

    def jacobian_t1(self, T, dT):
        """hnc3d.c:1289-1362: J dT = (chi-1)*(c'(t) dT) - dT."""
        if self._pool is not None:
            dc = np.empty_like(T)

            def clo(a, b):
                dc[:, a:b] = cl.closure1(self.closure, self.beta, self.v[:, a:b], T[:, a:b], dT[:, a:b])

            self._each_slab(clo)
            c_fft = self.fft(dc)
            t_fft = np.empty_like(c_fft)

            def oz(a, b):
                t_fft[:, a:b] = self._star_slab(c_fft[:, a:b] * self.h3, a, b)

            self._each_slab(oz)
            r = self.ifft(t_fft)

            def fin(a, b):
                r[:, a:b] *= 1.0 / self.L3
                r[:, a:b] -= dT[:, a:b]

            self._each_slab(fin)
            return r
        dc = cl.closure1(self.closure, self.beta, self.v, T, dT)
        t_fft = self.star(self.fft(dc) * self.h3)
        return self.ifft(t_fft) * (1.0 / self.L3) - dT

    def observables(self, T):
        """hnc3d.c:2157-2269: mu (native, HNC, KH, GF), PMV factor, g."""
        beta, rho = self.beta, self.rho
        c = cl.closure(self.closure, beta, self.v, T)
        h = c + T
        uc = coulomb_long(self.N, self.L, self.solute)
        clr = np.stack([0.0 + (-beta * self.charge[i]) * uc for i in range(self.m)])
        x = -beta * self.v + T

        def mu_of(method):
            dens = np.zeros(T.shape[1:])
            for i in range(self.m):
                dens = dens + cl.form(method, x[i], h[i], c[i], clr[i])
            return rho * dens.sum() * self.h3 / beta

        mu = mu_of(self.closure)
        mus = {"HNC": mu_of(cl.HNC), "KH": mu_of(cl.KH), "GF": mu_of(cl.PY)}
        pmv = 1 - sum(c[i].sum() * (rho * self.h3) for i in range(self.m))
        return {"mu": mu, "mu_all": mus, "pmv": pmv, "g": h + 1.0, "c": c, "h": h,
                "uc": uc, "x": x, "cl": clr}


def solute_solve(N, L, beta, rho, closure, solvent, solute, chi, rmax, renorm=True,
                 tol=1e-12, T0=None, picard_steps=0, verbose=False, chi3=None):
    """hnc3d_solute_solve (hnc3d.c:1762-2350) returning mu, PMV, g, T."""
    P = Problem(N, L, beta, rho, closure, solvent, solute, chi, rmax, renorm, chi3=chi3)
    T0 = np.zeros((P.m, P.N[2], P.N[1], P.N[0])) if T0 is None else T0
    jv = P.jacobian_t1 if closure != cl.PY else None
    T, iters = newton.solve(P.iterate_t1, T0, jv=jv, tol=tol, picard_steps=picard_steps,
                            verbose=verbose)
    out = P.observables(T)
    out["T"] = T
    out["iters"] = iters
    out["problem"] = P
    return out


def response(P, T, rtol=1e-12, sites=None):
    """Linear-response derivatives dmu/dR[n][3] at a converged T: the
    ``response`` branch of hnc3d_solute_solve (hnc3d.c:1969-2135) with
    response_t1 (hnc3d.c:1366-1421).

    Per unit displacement of site u along dim: dv = field1 (bgy3d-solutes.c:
    381-468, LJ plus the full capped Coulomb); B = beta (chi-1) * (f'(x) dv),
    the flagged jacobian_t1 (hnc3d.c:1305-1330); J dT = B solved from zero;
    dx = -beta dv + dT, dc = closure1(dx) - beta dv, dh = dc + dT; then
    chempot1 (hnc3d.c:627-650) with cl = -beta q_i uc held fixed.  ``sites``
    limits the rows computed (the others stay zero)."""
    beta, rho = P.beta, P.rho
    obs = P.observables(T)
    x, h, c, clr = obs["x"], obs["h"], obs["c"], obs["cl"]
    d = cl.closure_slope(P.closure, beta, P.v, T)
    shape = T.shape
    n = T.size
    A = sla.LinearOperator((n, n), matvec=lambda v: P.jacobian_t1(T, v.reshape(shape)).ravel(),
                           dtype=np.float64)
    dE = np.zeros((len(P.solute), 3))
    for u in (range(len(P.solute)) if sites is None else sites):
        for dim in range(3):
            dv = solute_field1(P.N, P.L, P.solvent, P.solute, u, dim)
            B = beta * P.ifft(P.star(P.fft(d * dv + dv) * P.h3)) * (1.0 / P.L3)
            dT, info = sla.gmres(A, B.ravel(), rtol=rtol, atol=0.0, restart=60, maxiter=200)
            dT = dT.reshape(shape)
            dx = -beta * dv + dT
            dc = d * dx - beta * dv
            dh = dc + dT
            dens = np.zeros(shape[1:])
            for i in range(P.m):
                dens = dens + cl.form1(P.closure, x[i], dx[i], h[i], dh[i], c[i], dc[i], clr[i])
            dE[u, dim] = rho * dens.sum() * P.h3 / beta
    return dE
