"""Site tables and synthetic solutes.

Sites are dicts {"name", "x": (3,), "sigma" (A), "epsilon" (kcal/mol),
"charge" (e)} -- the fields of ``Site`` (bgy3d-solutes.h:9-16).

The molecule entries restate the parameters of the reference's molecule
database (guile/solutes.scm:312-320 for water, 598-606 for the JC08 ions,
where ``(r0 (A x))`` means sigma = x * 2^(5/6), guile/molecule.scm:89-91).
"""
import numpy as np

_S56 = 2.0 ** (5.0 / 6.0)


def _water(h_sigma, h_eps):
    return [
        dict(name="O", x=(-0.288675134594813, 0.0, 0.0), sigma=3.1656, epsilon=0.1553, charge=-0.8476),
        dict(name="OH", x=(0.288675134594813, 0.816496580927726, 0.0), sigma=h_sigma, epsilon=h_eps,
             charge=0.4238),
        dict(name="OH", x=(0.288675134594813, -0.816496580927726, 0.0), sigma=h_sigma, epsilon=h_eps,
             charge=0.4238),
    ]


def _ion(name, r0, eps, q):
    return [dict(name=name, x=(0.0, 0.0, 0.0), sigma=r0 * _S56, epsilon=eps, charge=q)]


MOLECULES = {
    "water, PR-SPC/E": _water(0.4, 0.046),
    "water, cSPC/E": _water(1.1658, 0.01553),
    "Li+, JC08, SPC/E": _ion("Li", 0.791, 0.3367344, 1.0),
    "Na+, JC08, SPC/E": _ion("Na", 1.212, 0.3526418, 1.0),
    "K+, JC08, SPC/E": _ion("K", 1.593, 0.4297054, 1.0),
    "Rb+, JC08, SPC/E": _ion("Rb", 1.737, 0.4451036, 1.0),
    "Cs+, JC08, SPC/E": _ion("Cs", 2.021, 0.0898565, 1.0),
    "F-, JC08, SPC/E": _ion("F", 2.257, 0.0074005, -1.0),
    "Cl-, JC08, SPC/E": _ion("Cl", 2.711, 0.0127850, -1.0),
    "Br-, JC08, SPC/E": _ion("Br", 2.751, 0.0269586, -1.0),
    "I-, JC08, SPC/E": _ion("I", 2.919, 0.0427845, -1.0),
}


def find_molecule(name):
    """Look up a molecule by its database name (guile/molecule.scm:148)."""
    return [dict(s) for s in MOLECULES[name]]


def synthetic_solute(n_sites, radius=6.0, seed=20261203, min_sep=1.2,
                     q_range=0.8, sigma_range=(2.5, 4.0), eps_range=(0.05, 0.3)):
    """Seeded neutral LJ+charge solute: n sites uniform in a ball of ``radius``
    with ``min_sep`` minimum separation (rejection sampling), charges
    U[-q_range, q_range] shifted to zero net charge, sigma and epsilon
    uniform in their ranges.  NumPy PCG64 with the given seed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = []
    tries = 0
    while len(pts) < n_sites:
        tries += 1
        if tries > 1_000_000:
            raise RuntimeError("cannot place sites")
        p = rng.uniform(-radius, radius, size=3)
        if np.dot(p, p) > radius * radius:
            continue
        if all(np.linalg.norm(p - q) >= min_sep for q in pts):
            pts.append(p)
    q = rng.uniform(-q_range, q_range, size=n_sites)
    q = q - q.mean()
    sig = rng.uniform(*sigma_range, size=n_sites)
    eps = rng.uniform(*eps_range, size=n_sites)
    return [dict(name=f"S{i}", x=tuple(float(v) for v in pts[i]), sigma=float(sig[i]),
                 epsilon=float(eps[i]), charge=float(q[i])) for i in range(n_sites)]
