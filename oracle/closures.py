"""Closures and chemical-potential integrands -- restatement of closures.f90.

Test infrastructure only (see oracle/__init__.py).

Closure numbering follows ``ClosureEnum`` (bgy3d.h:211-223):
HNC=0, KH=1, PY=2, PSE0..PSE7 = 3..10.
"""
import numpy as np

HNC, KH, PY = 0, 1, 2
PSE0 = 3
NAMES = {"HNC": 0, "KH": 1, "PY": 2, **{f"PSE{n}": 3 + n for n in range(8)}}


def order(method):
    """closures.f90:156-174 (HNC: infinite, KH: 1, PSE-n: n)."""
    if method == HNC:
        return 10 ** 9
    if method == KH:
        return 1
    if PSE0 <= method <= PSE0 + 7:
        return method - PSE0
    return -1


def exps1(n, x):
    """Truncated exponential series by Horner, closures.f90:191-236."""
    c = 1.0
    y = np.zeros_like(x)
    for k in range(n, 0, -1):
        y = x * y + c
        c = c * k
    return (x / c) * y


def pse(n, x):
    """expm1(x) for x < 0, else the n-term series (closures.f90:405-432)."""
    neg = x < 0.0
    return np.where(neg, np.expm1(np.where(neg, x, 0.0)), exps1(n, np.where(neg, 0.0, x)))


def closure(method, beta, v, t):
    """c = closure(beta*v, t), closures.f90:107-128, 248-256, 278-295, 322-333, 365-377."""
    bv = beta * v
    if method == HNC:
        return np.expm1(-bv + t) - t                       # closure_hnc 248-256
    if method == KH:
        x = -bv + t                                        # closure_kh 278-295
        return np.where(x <= 0.0, np.expm1(np.minimum(x, 0.0)) - t, -bv)
    if method == PY:
        return np.exp(-bv) * (1 + t) - 1 - t               # closure_py 322-333
    if PSE0 <= method <= PSE0 + 7:
        return pse(order(method), -bv + t) - t             # closure_pse 365-377
    raise ValueError("no such closure")


def closure1(method, beta, v, t, dt):
    """dc = closure'(t) dt, closures.f90:131-153, 259-267, 298-316, 380-402.

    PY has no differential in the reference (returns huge, 150-151)."""
    bv = beta * v
    x = -bv + t
    if method == HNC:
        return np.expm1(x) * dt
    if method == KH:
        return np.where(x <= 0.0, np.expm1(np.minimum(x, 0.0)) * dt, 0.0)
    if PSE0 <= method <= PSE0 + 7:
        return pse(order(method) - 1, x) * dt
    raise ValueError("closure has no differential")


def closure_slope(method, beta, v, t):
    """The factor d = dc/dt such that closure1 == d * dt (used by tests)."""
    return closure1(method, beta, v, t, np.ones_like(t))


def _factorial(n):
    out = 1
    for k in range(2, n + 1):
        out *= k
    return out


def form(method, x, h, c, cl):
    """beta*mu/rho density, closures.f90:574-612 (elemental ``form``)."""
    base = -c - h * (c + cl) / 2
    if method == HNC:
        return base + h ** 2 / 2
    if method == KH:
        return np.where(h < 0, base + h ** 2 / 2, base)
    if method == PY:                    # "GF" functional in print_chempot
        return base
    if PSE0 <= method <= PSE0 + 7:
        m = order(method) + 1
        mx = float(_factorial(m))
        return np.where(h < 0, base + h ** 2 / 2, base + (h ** 2 / 2 - x ** m / mx))
    raise ValueError("no such closure")


def form1(method, x, dx, h, dh, c, dc, cl):
    """Differential of ``form``, closures.f90:615-653."""
    base = -dc - dh * (c + cl) / 2 - h * dc / 2
    if method == HNC:
        return base + h * dh
    if method == KH:
        return np.where(h < 0, base + h * dh, base)
    if method == PY:
        return base
    if PSE0 <= method <= PSE0 + 7:
        n = order(method)
        nx = float(_factorial(n))
        return np.where(h < 0, base + h * dh, base + (h * dh - x ** n * dx / nx))
    raise ValueError("no such closure")
