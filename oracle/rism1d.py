"""1D RISM / DRISM for the pure solvent and a solute -- restatement of rism.f90.

Test infrastructure only (see oracle/__init__.py).

Sites are dicts {"x": (3,), "sigma", "epsilon", "charge"} (the ``Site``
struct, bgy3d-solutes.h:9-16).  Pair arrays are [m][m][nrad] (the C
layout the reference hands across its FFI, rism.f90:57-102).
"""
import numpy as np
import scipy.fft
import scipy.special

from . import closures as cl
from . import newton

EPSILON0INV = 331.84164          # units.f90:50, bgy3d.h:145
ALPHA = 1.2                      # units.f90:61, bgy3d-solvents.h:9
FT_FW = 1.0                      # fft.f90:19
FT_BW = (2 * np.pi) ** 3         # fft.f90:20


def mkgrid(rmax, nrad):
    """fft.f90:101-118: r_i = (i-1/2) dr, k_i = (i-1/2) dk, dr dk = pi/n."""
    dr = rmax / nrad
    dk = np.pi / rmax
    i = np.arange(1, nrad + 1, dtype=np.float64)
    return (2 * i - 1) * dr / 2, dr, (2 * i - 1) * dk / 2, dk


def fourier_rows(f):
    """fft.f90:121-170: radial 3D FT kernel via DST-IV (FFTW RODFT11).

    g(p) = DST4[f(j) * 2n(2j-1)](p) / (2p-1), dr = 1; callers scale by
    dr^3 / FT_FW or dk^3 / FT_BW."""
    n = f.shape[-1]
    p = np.arange(1, n + 1, dtype=np.float64)
    g = f * (2 * n * (2 * p - 1))
    g = scipy.fft.dst(g, type=4, axis=-1)
    return g * (1.0 / (2 * p - 1))


def integrate(f):
    """fft.f90 ``integrate``: 4 pi sum f_i (2i-1)^2/4, summed backwards."""
    n = f.shape[-1]
    i = np.arange(1, n + 1, dtype=np.float64)
    w = (2 * i - 1) ** 2 / 4
    return 4 * np.pi * np.sum((f * w)[..., ::-1], axis=-1)


def j0(x):
    """bessel.f90:36-58 (series for |x| < 0.5)."""
    x = np.asarray(x, dtype=np.float64)
    c1, c2, c3 = -1 / 6.0, 1 / 120.0, -1 / 5040.0
    c4, c5, c6 = 1 / 362880.0, -1 / 39916800.0, 1 / 6227020800.0
    y = x * x
    series = 1 + y * (c1 + y * (c2 + y * (c3 + y * (c4 + y * (c5 + y * c6)))))
    small = np.abs(x) < 0.5
    xs = np.where(small, 1.0, x)
    return np.where(small, series, np.sin(xs) / xs)


def j1(x):
    """bessel.f90:61-91 (series for |x| < 0.25)."""
    x = np.asarray(x, dtype=np.float64)
    c1, c2, c3 = -1 / 10.0, 1 / 280.0, -1 / 15120.0
    c4, c5 = 1 / 1330560.0, -1 / 172972800.0
    y = x * x
    series = x / 3 * (1 + y * (c1 + y * (c2 + y * (c3 + y * (c4 + y * c5)))))
    small = np.abs(x) < 0.25
    xs = np.where(small, 1.0, x)
    return np.where(small, series, (np.sin(xs) / xs - np.cos(xs)) / xs)


def lj(r):
    """rism.f90:2201-2215."""
    sr6 = 1 / r ** 6
    return 4 * sr6 * (sr6 - 1)


def coulomb_long_fourier(k, alpha):
    """rism.f90:2371-2383: 4 pi exp(-k^2/4a^2)/k^2, 0 at k = 0."""
    k = np.asarray(k, dtype=np.float64)
    ks = np.where(k == 0.0, 1.0, k)
    return np.where(k == 0.0, 0.0, 4 * np.pi * np.exp(-ks ** 2 / (4 * alpha ** 2)) / ks ** 2)


def coulomb_long(r, alpha):
    """rism.f90:2386-2404."""
    r = np.asarray(r, dtype=np.float64)
    rs = np.where(r == 0.0, 1.0, r)
    return np.where(r == 0.0, alpha * 2 / np.sqrt(np.pi), scipy.special.erf(alpha * rs) / rs)


def coulomb_short(r, alpha):
    """rism.f90:2407-2415."""
    return scipy.special.erfc(alpha * r) / r


def pair(a, b):
    """Lorentz-Berthelot, rism.f90:1323-1350."""
    return (a["sigma"] + b["sigma"]) / 2, np.sqrt(a["epsilon"] * b["epsilon"])


def force_field(asites, bsites, r, k):
    """rism.f90:2082-2162 (no custom force fields)."""
    n, m = len(asites), len(bsites)
    vr = np.zeros((n, m, r.size))
    vk = np.zeros((n, m, k.size))
    for j, b in enumerate(bsites):
        for i, a in enumerate(asites):
            qab = a["charge"] * b["charge"]
            sigma, epsilon = pair(a, b)
            if sigma != 0.0:
                vr[i, j] = epsilon * lj(r / sigma) + EPSILON0INV * qab * coulomb_short(r, ALPHA)
            else:
                vr[i, j] = EPSILON0INV * qab * coulomb_short(r, ALPHA)
            vk[i, j] = EPSILON0INV * qab * coulomb_long_fourier(k, ALPHA)
    return vr, vk


def force_field_long(asites, bsites, r):
    """rism.f90:2165-2198."""
    v = np.zeros((len(asites), len(bsites), r.size))
    for i, a in enumerate(asites):
        for j, b in enumerate(bsites):
            v[i, j] = a["charge"] * b["charge"] * EPSILON0INV * coulomb_long(r, ALPHA)
    return v


def omega_fourier(sites, k):
    """rism.f90:1994-2032: omega_ab(k) = j0(k r_ab)."""
    m = len(sites)
    w = np.zeros((m, m, k.size))
    for j in range(m):
        for i in range(m):
            rab = np.linalg.norm(np.asarray(sites[i]["x"]) - np.asarray(sites[j]["x"]))
            w[i, j] = j0(k * rab)
    return w


# ---------------------------------------------------------------- DRISM
def _dipole(sites):
    """drism.f90:125-137."""
    q = np.array([s["charge"] for s in sites])
    x = np.array([s["x"] for s in sites], dtype=np.float64)
    return (q[:, None] * x).sum(axis=0)


def _weights(sites):
    """drism.f90:140-154: sigma^3 normalised."""
    w = np.array([s["sigma"] for s in sites]) ** 3
    return w / w.sum()


def _center(sites):
    """drism.f90:157-184."""
    w = _weights(sites)
    x = np.array([s["x"] for s in sites], dtype=np.float64)
    return (w[:, None] * x).sum(axis=0)


def _eigv(t):
    e, u = np.linalg.eigh(t)
    return e, u


def _axes(sites):
    """drism.f90:187-225 (shape tensor eigenvectors)."""
    c = _center(sites)
    w = _weights(sites)
    t = np.zeros((3, 3))
    for s, site in enumerate(sites):
        d = np.asarray(site["x"]) - c
        t += w[s] * np.outer(d, d)
    _, u = _eigv(t)
    return u


def dipole_axes(sites):
    """drism.f90:228-342: local axes with z along the dipole."""
    m = _dipole(sites)
    m = m / np.linalg.norm(m)
    v = _axes(sites).copy()
    e = np.zeros(3)
    for j in range(3):
        v[:, j] = v[:, j] - m * np.dot(m, v[:, j])
        e[j] = np.dot(v[:, j], v[:, j])
    i = int(np.argmin(e))
    u = np.zeros((3, 3))
    k = 0
    for j in range(3):
        if j == i:
            continue
        u[:, k] = v[:, j]
        k += 1
    u[:, 2] = m
    u[:, 1] = u[:, 1] - u[:, 0] * np.dot(u[:, 0], u[:, 1]) / np.dot(u[:, 0], u[:, 0])
    for j in range(3):
        u[:, j] = u[:, j] / np.linalg.norm(u[:, j])
    c = _center(sites)
    w = _weights(sites)
    t = np.zeros((2, 2))
    for s, site in enumerate(sites):
        d = np.asarray(site["x"]) - c
        dxy = np.array([np.dot(d, u[:, 0]), np.dot(d, u[:, 1])])
        t += w[s] * np.outer(dxy, dxy)
    _, vv = _eigv(t)
    u[:, 0:2] = u[:, 0:2] @ vv
    return u


def local_coords(sites, u):
    """drism.f90:345-370."""
    c = _center(sites)
    return np.array([[np.dot(u[:, i], np.asarray(s["x"]) - c) for i in range(3)] for s in sites]).T


def dipole_density(beta, rho, sites):
    """drism.f90:20-41: y = 4 pi beta rho mu^2 / 9 (times 1/eps0)."""
    return 4 * np.pi * beta * EPSILON0INV * rho * np.linalg.norm(_dipole(sites)) ** 2 / 9


def dipole_correction(beta, rho, eps, sites, k):
    """drism.f90:373-474: x_ab(k) = f_a(k) h_c(k) f_b(k)."""
    s = 0.5
    x = local_coords(sites, dipole_axes(sites))
    m = len(sites)
    f = np.zeros((k.size, m))
    for i in range(m):
        d = x[:, i]
        f[:, i] = j0(k * d[0]) * j0(k * d[1]) * j1(k * d[2])
    y = dipole_density(beta, rho, sites)
    h = (eps - (1 + 3 * y)) / (rho * y) * np.exp(-(k * s) ** 2 / 4)
    xk = np.zeros((m, m, k.size))
    for j in range(m):
        for i in range(m):
            xk[i, j] = f[:, i] * h * f[:, j]
    return xk


# ------------------------------------------------------------- OZ solves
def oz_vv_equation_c_t(rho, C, W):
    """rism.f90:2432-2560.  C, W: [m][m][nrad]."""
    m = C.shape[0]
    if m == 1:
        c = C[0, 0]
        return (rho * (c * c) / (1 - rho * c))[None, None, :]
    Cp = np.moveaxis(C, -1, 0)
    Wp = np.moveaxis(W, -1, 0)
    H = Wp @ Cp
    T = np.eye(m)[None] - H * rho
    H = H @ Wp
    H = np.linalg.solve(T, H)
    return np.moveaxis(H - Cp, 0, -1)


def oz_uv_equation_c_t(c_uv, w_uu, x_vv):
    """rism.f90:2583-2607: t = w c x - c per k."""
    C = np.moveaxis(c_uv, -1, 0)
    W = np.moveaxis(w_uu, -1, 0)
    X = np.moveaxis(x_vv, -1, 0)
    return np.moveaxis(W @ (C @ X) - C, 0, -1)


def chempot(method, rmax, beta, rho, v, vl, t):
    """closures.f90 ``chempot``: mu = integrate(sum form) * rho dr^3 / beta."""
    nrad = t.shape[-1]
    dr = rmax / nrad
    c = cl.closure(method, beta, v, t)
    clr = -beta * vl
    h = c + t
    x = -beta * v + t
    dens = cl.form(method, x, h, c, clr).sum(axis=(0, 1))
    return integrate(dens) * (rho * dr ** 3 / beta)


def rism_vv(method, nrad, rmax, beta, rho, sites, eps=0.0, tol=1e-13, verbose=False):
    """rism.f90:310-583.  Returns dict with t, chi = w + rho h (m,m,nrad), mu."""
    r, dr, k, dk = mkgrid(rmax, nrad)
    m = len(sites)
    vr, vk = force_field(sites, sites, r, k)
    wk = omega_fourier(sites, k)
    xk = dipole_correction(beta, rho, eps, sites, k) if eps != 0.0 else np.zeros_like(wk)
    A = 1.0

    def iterate_t(t):
        c = cl.closure(method, beta, vr, t)
        c = fourier_rows(c) * (dr ** 3 / FT_FW)
        c = c - (beta * A) * vk
        if eps != 0.0:
            dt = oz_vv_equation_c_t(rho, c, wk + rho * xk) + xk
        else:
            dt = oz_vv_equation_c_t(rho, c, wk)
        dt = dt - (beta * A) * vk
        dt = fourier_rows(dt) * (dk ** 3 / FT_BW)
        return dt - t

    def iterate_rt(rt):                              # rism.f90:539-546
        return r * iterate_t(rt / r)

    rt, _ = newton.solve(iterate_rt, np.zeros((m, m, nrad)), tol=tol, verbose=verbose)
    t = rt / r
    c = cl.closure(method, beta, vr, t)
    h = fourier_rows(c + t) * (dr ** 3 / FT_FW)
    chi = wk + rho * h
    vl = force_field_long(sites, sites, r)
    mu = chempot(method, rmax, beta, rho, vr, vl, t)
    return {"t": t, "chi": chi, "mu": mu, "r": r, "k": k}


def rism_uv(method, nrad, rmax, beta, rho, solvent, chi, solute, tol=1e-13, verbose=False):
    """rism.f90:586-859 (ng = .false., no RBC).  Returns dict with t, mu."""
    r, dr, k, dk = mkgrid(rmax, nrad)
    v_uvr, v_uvk = force_field(solute, solvent, r, k)
    w_uuk = omega_fourier(solute, k)
    s_uvk = -beta * (oz_uv_equation_c_t(v_uvk, w_uuk, chi) + v_uvk)

    def iterate_t(t):
        c = cl.closure(method, beta, v_uvr, t)
        c = fourier_rows(c) * (dr ** 3 / FT_FW)
        dt = oz_uv_equation_c_t(c, w_uuk, chi) + s_uvk
        dt = fourier_rows(dt) * (dk ** 3 / FT_BW)
        return dt - t

    def jacobian_t(t, dt):
        c = cl.closure1(method, beta, v_uvr, t, dt)
        c = fourier_rows(c) * (dr ** 3 / FT_FW)
        ddt = oz_uv_equation_c_t(c, w_uuk, chi)
        ddt = fourier_rows(ddt) * (dk ** 3 / FT_BW)
        return ddt - dt

    jv = jacobian_t if method != cl.PY else None
    t, _ = newton.solve(iterate_t, np.zeros((len(solute), len(solvent), nrad)), jv=jv,
                        tol=tol, verbose=verbose)
    vl = force_field_long(solute, solvent, r)
    mu = chempot(method, rmax, beta, rho, v_uvr, vl, t)
    return {"t": t, "mu": mu}
