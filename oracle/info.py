"""Post-processing observables of a solute solve -- restatement of info()
and print_info() (bgy3d-potential.c:245-493) with bgy3d_solvent_field,
the FFT Poisson solve (bgy3d-poisson.c:103-183), the Gaussian core density
cores() (bgy3d-solutes.c:555-577), the trigonometric interpolation
bgy3d_fft_interp (bgy3d-fftw3.c:504-612) and the grid moments
bgy3d_moments (bgy3d-vec.c:476-593).

Test infrastructure only (see oracle/__init__.py).

Fields are [N2][N1][N0] arrays on the centred grid r = i h - L/2.
"""
import numpy as np
import scipy.fft

from .hnc3d import G, coulomb_long, kfreq, rgrid
from .rism1d import EPSILON0INV


def moments(v, N, L):
    """bgy3d_moments: 0th, 1st and 2nd moments of v about the grid index
    N/2 (not the box centre; vec_moments1/2 take i - 0.5 N), scaled by the
    volume element and the spacings.  v is [N2][N1][N0]."""
    h = [L[d] / N[d] for d in range(3)]
    dV = h[0] * h[1] * h[2]
    c = [np.arange(N[d]) - 0.5 * N[d] for d in range(3)]
    X = [c[0][None, None, :], c[1][None, :, None], c[2][:, None, None]]
    q = dV * v.sum()
    d = np.array([dV * h[a] * (v * X[a]).sum() for a in range(3)])
    Q = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            Q[a, b] = dV * h[a] * h[b] * (v * X[a] * X[b]).sum()
    return q, d, Q


def g_moments(g, N, L):
    """The regression summary's moments of a distribution (the ``moments``
    command, guile/bgy3d.scm:1136-1155): bgy3d_moments of 1 - g."""
    return moments(1.0 - g, N, L)


def cores(N, L, solute, alpha=G):
    """Gaussian solute charge density (G/sqrt(pi))^3 sum q e^{-G^2 r^2}."""
    x, y, z = rgrid(N, L)
    s = np.zeros((N[2], N[1], N[0]))
    for b in solute:
        bx = b["x"]
        r2 = (x - bx[0]) ** 2 + (y - bx[1]) ** 2 + (z - bx[2]) ** 2
        s = s + b["charge"] * np.exp(-alpha ** 2 * r2)
    return (alpha / np.sqrt(np.pi)) ** 3 * s


def poisson_fft(rho, N, L):
    """bgy3d_poisson with q = -4 pi/eps0: u(k) = 4 pi/eps0 h^3 rho(k) / k^2,
    u(0) = 0, on the r2c half grid (unnormalised, the reference's ve_fft)."""
    h = [L[d] / N[d] for d in range(3)]
    dk = [2 * np.pi / L[d] for d in range(3)]
    k0 = (kfreq(np.arange(N[0] // 2 + 1), N[0]) * dk[0])[None, None, :]
    k1 = (kfreq(np.arange(N[1]), N[1]) * dk[1])[None, :, None]
    k2 = (kfreq(np.arange(N[2]), N[2]) * dk[2])[:, None, None]
    kq = k2 ** 2 + k1 ** 2 + k0 ** 2
    scale = 4 * np.pi * EPSILON0INV * h[0] * h[1] * h[2]
    fac = np.where(kq != 0.0, scale / np.where(kq != 0.0, kq, 1.0), 0.0)
    return scipy.fft.rfftn(rho, axes=(-3, -2, -1)) * fac


def fft_interp(Y, N, pts):
    """bgy3d_fft_interp: trigonometric interpolation of the half-spectrum Y
    at fractional grid coordinates pts[p][3] (x fastest in Y[z][y][x])."""
    out = np.zeros(len(pts))
    kk = [np.arange(N[0] // 2 + 1), np.arange(N[1]), np.arange(N[2])]
    for p, x in enumerate(pts):
        w = []
        for d in range(3):
            k = kk[d]
            K = kfreq(k, N[d])
            ph = (2 * np.pi / N[d]) * K * x[d]
            nyq = (N[d] - 2 * k) % N[d] == 0
            w.append(np.where(nyq, np.cos(ph) + 0j, np.exp(1j * ph)))
        wk = w[0][None, None, :] * w[1][None, :, None] * w[2][:, None, None]
        K0 = kfreq(kk[0], N[0])
        half = np.where((N[0] - 2 * K0) % N[0] == 0, 0.5, 1.0)[None, None, :]
        out[p] = np.sum(2 * np.real(Y * wk * half)) / (N[0] * N[1] * N[2])
    return out


def trilinear(v, N, pts):
    """bgy3d_interp (bgy3d-interp.c:37-136): trilinear interpolation of the
    real field v[N2][N1][N0] at fractional grid coordinates, periodic."""
    out = np.zeros(len(pts))
    for p, r in enumerate(pts):
        i0 = [int(np.floor(r[d])) for d in range(3)]
        f = [r[d] - i0[d] for d in range(3)]
        s = 0.0
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    w = (f[0] if dx else 1 - f[0]) * (f[1] if dy else 1 - f[1]) * (f[2] if dz else 1 - f[2])
                    s += w * v[(i0[2] + dz) % N[2], (i0[1] + dy) % N[1], (i0[0] + dx) % N[0]]
        out[p] = s
    return out


def info(N, L, rho, solvent, solute, g):
    """The observables print_info writes for the regression summary:
    charges, dipoles and second moments of the solute (rho_u) and solvent
    (rho_v = rho sum_i q_i g_i) charge densities, the cores' dipole, and
    <U_v|rho_N>, <U_v|rho_u>, <rho_v|U_u>.  g: [m][N2][N1][N0].

    <U_v|rho_N> takes the solvent potential at the solute sites; the
    shipped bgy3d_pot_interp interpolates trigonometrically
    (bgy3d-potential.c:125-143), while the regression outputs
    (test/out/*.hnc3d.g1) hold the trilinear value of bgy3d_interp
    (bgy3d-interp.c): both are returned."""
    h = [L[d] / N[d] for d in range(3)]
    h3 = h[0] * h[1] * h[2]
    L3 = L[0] * L[1] * L[2]
    rho_v = np.zeros(g.shape[1:])
    for i, a in enumerate(solvent):
        rho_v = rho_v + a["charge"] * rho * g[i]
    ve_fft = poisson_fft(rho_v, N, L)
    ve = scipy.fft.irfftn(ve_fft, s=(N[2], N[1], N[0]), axes=(-3, -2, -1)) * (N[0] * N[1] * N[2]) / L3
    rho_u = cores(N, L, solute)
    uc = coulomb_long(N, L, solute)
    qu, du, Qu = moments(rho_u, N, L)
    qv, dv, Qv = moments(rho_v, N, L)
    dn = np.zeros(3)
    for b in solute:
        dn = dn + b["charge"] * np.asarray(b["x"])
    pts = [[(b["x"][d] + L[d] / 2) / h[d] for d in range(3)] for b in solute]
    vfft = scipy.fft.rfftn(ve, axes=(-3, -2, -1))
    vs = fft_interp(vfft, N, pts)
    vl = trilinear(ve, N, pts)
    val1 = float(sum(b["charge"] * vs[i] for i, b in enumerate(solute)))
    val1l = float(sum(b["charge"] * vl[i] for i, b in enumerate(solute)))
    return {"q_u": qu, "d_u": du, "Q_u": Qu, "q_v": qv, "d_v": dv, "Q_v": Qv, "d_n": dn,
            "U_v_rho_N": val1, "U_v_rho_N_trilinear": val1l, "U_v_rho_u": h3 * float(np.sum(ve * rho_u)),
            "rho_v_U_u": h3 * float(np.sum(uc * rho_v)), "site_potential": vs, "site_potential_trilinear": vl}
