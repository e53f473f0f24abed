"""Newton-GMRES stand-in for PETSc SNESNEWTONLS/KSPGMRES (bgy3d-snes.c:160-346).

Test infrastructure only (see oracle/__init__.py).

The reference drives iterate_t1/jacobian_t1 with SNES NEWTONLS, a shell
Jacobian, GMRES(30) without preconditioner and KSP rtol = 100 * 1e-5
(bgy3d-snes.c:243, 277, 306).  Only the fixed point matters for parity,
so this driver is a plain inexact Newton with backtracking on ||F||_2,
optionally preceded by damped Picard steps (``bgy3d_snes_trial``,
bgy3d-snes.c:387-399: 100 steps at lambda = 0.02).
"""
import numpy as np
import scipy.sparse.linalg as sla


class NotConverged(RuntimeError):
    pass


def solve(F, x0, jv=None, tol=1e-12, max_iter=200, krylov_rtol=1e-3,
          restart=30, picard_steps=0, picard_lambda=0.02, verbose=False):
    """Find x with ||F(x)||_inf < tol.

    F(x) -> residual (same shape as x).  jv(x, v) -> J(x) v; if None a
    central finite difference of F is used.
    """
    x = np.array(x0, dtype=np.float64, copy=True)
    shape = x.shape
    for _ in range(picard_steps):                    # bgy3d_snes_picard 348-384
        dx = F(x)
        x += picard_lambda * dx
        if np.max(np.abs(dx)) < tol:
            return x, 0
    f = F(x)
    n = x.size
    for it in range(max_iter):
        finf = np.max(np.abs(f))
        if verbose:
            print(f"  newton {it}: |F|inf={finf:.3e} |F|2={np.linalg.norm(f):.3e}")
        if finf < tol:
            return x, it
        if jv is None:
            def mv(v, x=x):
                v = v.reshape(shape)
                nv = np.linalg.norm(v)
                if nv == 0:
                    return np.zeros(n)
                eps = 1e-7 * max(1.0, np.linalg.norm(x)) / nv
                return ((F(x + eps * v) - F(x - eps * v)) / (2 * eps)).ravel()
        else:
            def mv(v, x=x):
                return jv(x, v.reshape(shape)).ravel()
        A = sla.LinearOperator((n, n), matvec=mv, dtype=np.float64)
        dx, info = sla.gmres(A, -f.ravel(), rtol=krylov_rtol, restart=restart,
                             maxiter=max(1, 1000 // restart), atol=0.0)
        dx = dx.reshape(shape)
        f2 = np.dot(f.ravel(), f.ravel())
        lam = 1.0
        for _ in range(30):                          # backtracking on ||F||_2
            xn = x + lam * dx
            fn = F(xn)
            fn2 = np.dot(fn.ravel(), fn.ravel())
            if fn2 <= (1.0 - 1e-4 * lam) * f2 or fn2 == 0.0:
                break
            lam *= 0.5
        x, f = xn, fn
    if np.max(np.abs(f)) < tol:
        return x, max_iter
    raise NotConverged(f"no convergence: |F|inf = {np.max(np.abs(f)):.3e}")


def jager(F, x0, lam, max_iter, tol):
    """bgy3d_snes_jager (bgy3d-snes.c:402-509): x += a F(x) with the mixing
    coefficient a = a1 every 10th iteration ("moves"), lambda otherwise; a1
    doubles (up to 1) after 20 quiet iterations and halves back (not below
    lambda) when a move made an otherwise falling norm go up.  Returns
    (x, iterations, last |F|inf)."""
    x = np.array(x0, dtype=np.float64, copy=True)
    a0 = a1 = lam
    norm_old = 0.0
    mycount = upwards = 0
    nth = 10
    norm = np.inf
    for it in range(max_iter):
        dx = F(x)
        norm = float(np.max(np.abs(dx)))
        a = a1 if it % nth == 0 else a0
        x += a * dx
        up = norm > norm_old
        norm_old = norm
        mycount += 1
        if it % nth != 1:
            upwards = 1 if up else 0
        if it % nth == 1 and up and upwards == 0 and it > 2 * nth:
            a1 = max(a1 / 2.0, a0)
            mycount = 0
        if mycount > 2 * nth:
            a1 = min(a1 * 2.0, 1.0)
            mycount = 0
        if norm <= tol:
            return x, it + 1, norm
    return x, max_iter, norm
