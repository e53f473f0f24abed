"""The x-axis grid transfers of the two-grid preconditioner with both sides
by FFT (k_restrict_fx2 / k_prolong_fx2), restated step by step in NumPy:
the packed half-length transforms and their untangle / pack twiddles give
the dense band-limited restriction R and prolongation P that the library
tabulates for the other axes (s(x) = sum_{|k|<=K} w_k cos(2 pi k x),
w_{+-K} = 1/2, R = s / nf, P = s / nc)."""
import numpy as np
import pytest


def dense_ops(nf, nc):
    K = nc // 2
    i = np.arange(nc)[:, None]
    j = np.arange(nf)[None, :]
    x = (i * nf - j * nc) % (nc * nf) / (nc * nf)
    s = np.ones_like(x) + 2 * sum(np.cos(2 * np.pi * k * x) for k in range(1, K)) + np.cos(2 * np.pi * K * x)
    return s / nf, (s / nc).T  # R [nc][nf], P [nf][nc]


def r2c_packed(x):
    """X_0..X_M of a real row of 2M points from the M-point complex FFT of
    z_j = x_2j + i x_2j+1 and the untangle X_k = E_k + e^{-2 pi i k / 2M} O_k."""
    M = x.size // 2
    Z = np.fft.fft(x[0::2] + 1j * x[1::2])
    k = np.arange(M + 1)
    zk, zm = Z[k % M], Z[(M - k) % M]
    E, O = (zk + np.conj(zm)) / 2, (zk - np.conj(zm)) / 2j
    return E + np.exp(-2j * np.pi * k / (2 * M)) * O


def c2r_packed(X, M):
    """Unnormalised real inverse of length 2M from X_0..X_K (zero above K,
    Im X_0 and Im X_M dropped): the packed Z_k and an M-point inverse FFT."""
    Xf = np.zeros(M + 1, complex)
    Xf[:min(M, X.size - 1) + 1] = X[:M + 1]
    Xf[0] = Xf[0].real
    Xf[M] = Xf[M].real
    k = np.arange(M)
    xk, xm = Xf[k], np.conj(Xf[M - k])
    Z = (xk + xm) + 1j * np.exp(1j * np.pi * k / M) * (xk - xm)
    z = np.fft.ifft(Z) * M
    out = np.empty(2 * M)
    out[0::2], out[1::2] = z.real, z.imag
    return out


@pytest.mark.parametrize("nf, nc", [(256, 64), (512, 128), (128, 48), (96, 48), (64, 48)])
def test_restriction_by_packed_transforms(nf, nc):
    R, _ = dense_ops(nf, nc)
    x = np.random.default_rng(nf + nc).standard_normal(nf)
    X = r2c_packed(x)
    assert np.allclose(X, np.fft.rfft(x), atol=1e-10)
    K = nc // 2
    out = c2r_packed(X[:K + 1], nc // 2) / nf
    assert np.max(np.abs(out - R @ x)) < 1e-12 * np.max(np.abs(R @ x)) * nf


@pytest.mark.parametrize("nf, nc", [(256, 64), (512, 128), (128, 48), (96, 48), (64, 48)])
def test_prolongation_by_packed_transforms(nf, nc):
    _, P = dense_ops(nf, nc)
    y = np.random.default_rng(nf * nc).standard_normal(nc)
    K = nc // 2
    Y = r2c_packed(y)
    f = np.full(K + 1, 1.0 / nc)
    f[K] = 0.5 / nc
    out = c2r_packed(Y * f, nf // 2)
    assert np.max(np.abs(out - P @ y)) < 1e-12 * np.max(np.abs(P @ y)) * nf
