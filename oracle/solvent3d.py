"""3D-RISM of the pure solvent -- restatement of hnc3d_solvent_solve
(hnc3d.c:803-1073) with iterate_t2 (hnc3d.c:353-456) and the OZ solve
compute_t2_m (hnc3d.c:231-323).

Test infrastructure only (see oracle/__init__.py).

The unknowns are the m(m+1)/2 site-site indirect correlations t_ij (i >= j),
packed in the order of vec_aliases_create2 (bgy3d-vec.h:739-758): pair
p = i(i+1)/2 + j, each a real field [N2][N1][N0] centred on the box (r =
i h - L/2).  k-space quantities are on the r2c half grid [N2][N1][N0/2+1]
as in oracle.hnc3d.

Per k the OZ equation of the molecular solvent is solved for the full
h = (1 - rho W C)^-1 W C W and t = h - c (the column-major zgemm / zgesv
sequence of compute_t2_m reduces to this for the symmetric W and C); the
m = 1 branch of the reference (compute_t2_1, hnc3d.c:215-224) writes to
t[n] instead of t[i] and is not restated -- the general formula with W = 1
serves every m.
"""
import numpy as np
import scipy.fft
import scipy.sparse.linalg as sla
import scipy.special

from . import closures as cl
from . import newton
from .hnc3d import G, interp, kabs, kgrid, rgrid
from .rism1d import EPSILON0INV, rism_vv

CUTOFF = 1.0e8                  # bgy3d-force.h:10
CUTOFF2 = CUTOFF * 1.0e-5       # bgy3d-force.h:11
_WORKERS = 8


def npairs(m):
    return m * (m + 1) // 2


def pairs(m):
    """(p, i, j) for i >= j in packing order."""
    out = []
    for i in range(m):
        for j in range(i + 1):
            out.append((len(out), i, j))
    return out


def lennard_jones(r, epsilon, sigma):
    """bgy3d-force.h:30-44 (capped at epsilon * CUTOFF)."""
    r = np.asarray(r, dtype=np.float64)
    if sigma == 0.0 or epsilon == 0.0:
        return np.zeros_like(r)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        sr = sigma / r
        sr6 = (sr * sr) * (sr * sr) * (sr * sr)
        re = 4 * epsilon * sr6 * (sr6 - 1)
    return np.where(np.abs(re) > epsilon * CUTOFF, epsilon * CUTOFF, re)


def coulomb_short(r, q2, alpha=G):
    """bgy3d-force.h:87-98 (the non-negative erfc(G r)/r capped at CUTOFF2)."""
    r = np.asarray(r, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        f = scipy.special.erfc(alpha * r) / r
    return np.where(f > CUTOFF2, EPSILON0INV * q2 * CUTOFF2, EPSILON0INV * q2 * f)


def coulomb_long_fourier(k, q2, alpha=G):
    """bgy3d-force.h:139-148: (4 pi/eps0) q2 exp(-k^2/4G^2)/k^2, 0 at k = 0."""
    k2 = k * k
    ks = np.where(k2 == 0.0, 1.0, k2)
    return np.where(k2 == 0.0, 0.0, (4 * np.pi * EPSILON0INV) * q2 * np.exp(-k2 / (4 * alpha ** 2)) / ks)


class SolventProblem:
    """Everything hnc3d_solvent_solve sets up before SNES (hnc3d.c:854-925)."""

    def __init__(self, N, L, beta, rho, closure, solvent):
        self.N = tuple(int(n) for n in N)
        self.L = tuple(float(x) for x in L)
        self.h = tuple(self.L[d] / self.N[d] for d in range(3))
        self.h3 = self.h[0] * self.h[1] * self.h[2]
        self.L3 = self.L[0] * self.L[1] * self.L[2]
        self.beta, self.rho, self.closure = float(beta), float(rho), int(closure)
        self.solvent = solvent
        self.m = m = len(solvent)
        self.P = pairs(m)
        x, y, z = rgrid(self.N, self.L)
        r = np.sqrt((x * x + y * y) + z * z)   # vec_rmap (bgy3d-vec.h:646-654)
        kk = kabs(self.N, self.L)
        _, _, _, sign = kgrid(self.N, self.L)
        self.sign = sign                       # bgy3d_vec_fft_trans (bgy3d-vec.c:618-646)
        self.v = np.zeros((npairs(m),) + r.shape)
        self.vl = np.zeros((npairs(m),) + kk.shape)   # v_long_fft, centred (real)
        for p, i, j in self.P:                 # bgy3d_pair_potential (bgy3d-force.c:123-147)
            a, b = solvent[i], solvent[j]
            eps = np.sqrt(a["epsilon"] * b["epsilon"])
            sig = 0.5 * (a["sigma"] + b["sigma"])
            q2 = a["charge"] * b["charge"]
            self.v[p] = lennard_jones(r, eps, sig) + coulomb_short(r, q2)
            self.vl[p] = coulomb_long_fourier(kk, q2) * sign
        # omega_intra (bgy3d-pure.c:241-276): sinc(2 pi r_ij / L |n|), corner
        i0 = np.arange(self.N[0] // 2 + 1)
        i1, i2 = np.arange(self.N[1]), np.arange(self.N[2])
        from .hnc3d import kfreq
        n2 = (kfreq(i0, self.N[0]) ** 2)[None, None, :] + (kfreq(i1, self.N[1]) ** 2)[None, :, None] + \
             (kfreq(i2, self.N[2]) ** 2)[:, None, None]
        nk = np.sqrt(n2.astype(np.float64))
        self.W = np.zeros((m, m) + kk.shape)
        for i in range(m):
            self.W[i, i] = 1.0
            for j in range(i):
                d = np.linalg.norm(np.asarray(solvent[i]["x"]) - np.asarray(solvent[j]["x"]))
                kr = (2.0 * np.pi * d / self.L[0]) * nk
                krs = np.where(kr == 0.0, 1.0, kr)
                w = np.where(kr == 0.0, 1.0, np.sin(krs) / krs)
                self.W[i, j] = self.W[j, i] = w

    def fft(self, x):
        return scipy.fft.rfftn(x, axes=(-3, -2, -1), workers=_WORKERS)

    def ifft(self, y):
        n = self.N[0] * self.N[1] * self.N[2]
        return scipy.fft.irfftn(y, s=(self.N[2], self.N[1], self.N[0]), axes=(-3, -2, -1), workers=_WORKERS) * n

    def full(self, packed):
        """[npairs][...] -> symmetric [...][m][m]."""
        m = self.m
        out = np.zeros(packed.shape[1:] + (m, m), dtype=packed.dtype)
        for p, i, j in self.P:
            out[..., i, j] = packed[p]
            out[..., j, i] = packed[p]
        return out

    def ck(self, T):
        """c(t) in k-space at the grid corner, long range included
        (hnc3d.c:382-405): C = [FFT(c) h^3 - beta v_long] * sign."""
        c = cl.closure(self.closure, self.beta, self.v, T)
        return (self.fft(c) * self.h3 - self.beta * self.vl) * self.sign

    def oz(self, Cp):
        """compute_t2_m (hnc3d.c:231-323): X = (1 - rho W C)^-1 W C W per k."""
        m = self.m
        C = self.full(Cp)
        W = np.moveaxis(self.W, (0, 1), (-2, -1)).astype(complex)
        WC = W @ C
        A = np.eye(m)[None, None, None] - self.rho * WC
        X = np.linalg.solve(A, WC @ W)
        return C, W, A, X

    def back(self, Tk):
        """t-space of a packed corner k-field (hnc3d.c:411-437)."""
        t = Tk * self.sign - self.beta * self.vl
        return self.ifft(t) * (1.0 / self.L3)

    def iterate_t2(self, T):
        """hnc3d.c:353-456: dT = t[T] - T."""
        C, W, A, X = self.oz(self.ck(T))
        Tk = np.stack([X[..., i, j] - C[..., i, j] for _, i, j in self.P])
        return self.back(Tk) - T

    def jacobian_t2(self, T, dT):
        """Differential of iterate_t2 (the reference has none, "FIXME: no
        Jacobian yet!"; SNES then differentiates F itself): with A X = W C W,
        dX = A^-1 W dC (W + rho X)."""
        if getattr(self, "_jT", None) is not T:      # one OZ factorisation per Newton step
            self._jT, self._jOZ = T, self.oz(self.ck(T))
        C, W, A, X = self._jOZ
        dc = cl.closure1(self.closure, self.beta, self.v, T, dT)
        dC = self.full(self.fft(dc) * self.h3 * self.sign)
        dX = np.linalg.solve(A, W @ dC @ (W + self.rho * X))
        dTk = np.stack([dX[..., i, j] - dC[..., i, j] for _, i, j in self.P])
        return self.ifft(dTk * self.sign) * (1.0 / self.L3) - dT

    def initial_guess(self, nrad=None, rmax=None, tol=1e-10):
        """The 1D RISM t(r) on the upscaled grid tabulated on the 3D grid
        (hnc3d.c:824-851, upscale 776-787: rmax = 2 max(L), nrad = 16 max(N))."""
        rmax = 4 * max(self.L) / 2 if rmax is None else rmax
        nrad = 16 * max(self.N) if nrad is None else nrad
        one = rism_vv(self.closure, nrad, rmax, self.beta, self.rho, self.solvent, tol=tol)
        x, y, z = rgrid(self.N, self.L)
        r = np.sqrt((x * x + y * y) + z * z)
        T = np.zeros((npairs(self.m),) + r.shape)
        for p, i, j in self.P:
            T[p] = interp(r, one["t"][i, j], rmax / nrad)   # vec_rtab (bgy3d-vec.c:49-56)
        return T

    def observables(self, T):
        """Post-processing of hnc3d_solvent_solve (hnc3d.c:958-1066): mu for
        the HNC / KH / GF functionals over all m x m pairs (print_chempot,
        hnc3d.c:674-694), the compressibility (print_kappa, 738-760), chi - 1
        on the k grid (the x%d%d-fft.bin content, 1020-1048) and g."""
        beta, rho = self.beta, self.rho
        c = cl.closure(self.closure, beta, self.v, T)
        h = c + T
        clr = np.stack([self.ifft(self.vl[p]) * (-beta / self.L3) for p, _, _ in self.P])
        x = -beta * self.v + T
        mult = np.array([1.0 if i == j else 2.0 for _, i, j in self.P])

        def mu_of(method):
            s = 0.0
            for p, _, _ in self.P:
                s += mult[p] * cl.form(method, x[p], h[p], c[p], clr[p]).sum()
            return rho * s * self.h3 / beta

        c0 = sum(mult[p] * c[p].sum() for p, _, _ in self.P) * (rho * self.h3)
        chi = np.zeros((npairs(self.m),) + self.W.shape[2:], dtype=complex)
        for p, i, j in self.P:
            chi[p] = self.fft(rho * h[p]) * self.h3 * self.sign
            if i != j:
                chi[p] += self.W[i, j]
        return {"mu": mu_of(self.closure), "mu_all": {"HNC": mu_of(cl.HNC), "KH": mu_of(cl.KH), "GF": mu_of(cl.PY)},
                "a": c0 / 2 / beta, "kappa": beta / (1 - c0) / rho, "chi_fft": chi, "g": h + 1.0, "c": c, "h": h}


def solvent_solve(N, L, beta, rho, closure, solvent, tol=1e-12, T0=None, verbose=False):
    """hnc3d_solvent_solve (hnc3d.c:803-1073) returning mu, kappa, chi - 1 (k
    grid, packed pairs), g and T."""
    P = SolventProblem(N, L, beta, rho, closure, solvent)
    if T0 is None:
        T0 = P.initial_guess()
    T, iters = newton.solve(P.iterate_t2, T0, jv=P.jacobian_t2, tol=tol, verbose=verbose)
    out = P.observables(T)
    out["T"] = T
    out["iters"] = iters
    out["problem"] = P
    return out
