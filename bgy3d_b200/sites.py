"""Site tables and synthetic solutes.

Sites are dicts {"name", "x": (3,), "sigma" (A), "epsilon" (kcal/mol),
"charge" (e)} -- the fields of ``Site`` (bgy3d-solutes.h:9-16).

The molecule entries restate the parameters of the reference's molecule
database (guile/solutes.scm:312-320 for water, 598-606 for the JC08 ions,
and the molecules of its regression tests, cited per entry,
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


def _mol(rows):
    return [dict(name=n, x=tuple(x), sigma=s, epsilon=e, charge=q) for n, x, s, e, q in rows]


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
    # guile/solutes.scm:252-255
    "water": _mol([("O", (-0.2929, 0.0, 0.0), 3.1506, 0.1521, -0.834),
                   ("OH", (0.2929, 0.757, 0.0), 0.4, 0.046, 0.417),
                   ("OH", (0.2929, -0.757, 0.0), 0.4, 0.046, 0.417)]),
    # guile/solutes.scm:127-129
    "hydrogen chloride": _mol([("H", (0.6285, 0.0, 0.0), 2.735, 0.03971, 0.2),
                               ("Cl", (-0.6285, 0.0, 0.0), 3.353, 0.51434, -0.2)]),
    # guile/solutes.scm:147-150
    "carbon disulfide": _mol([("C", (0.0, 0.0, 0.0), 3.2, 0.10128, -0.308),
                              ("S1", (-1.56, 0.0, 0.0), 3.52, 0.395, 0.154),
                              ("S2", (1.56, 0.0, 0.0), 3.52, 0.395, 0.154)]),
    # guile/solutes.scm:408-414
    "methanol": _mol([("C", (-0.748, -0.015, 0.024), 3.5, 0.066, 0.145),
                      ("HC1", (-1.293, -0.202, -0.901), 2.5, 0.03, 0.04),
                      ("HC2", (-1.263, 0.754, 0.6), 2.5, 0.03, 0.04),
                      ("HC3", (-0.699, -0.934, 0.609), 2.5, 0.03, 0.04),
                      ("O", (0.558, 0.42, -0.278), 3.12, 0.17, -0.683),
                      ("OH", (0.716, 1.404, 0.137), 0.4, 0.04, 0.418)]),
    # guile/solutes.scm:420-436
    "butanoic acid": _mol([("C1", (1.422, -0.017, 0.0), 3.75, 0.105, 0.52),
                           ("O1", (1.422, 1.353, 0.0), 2.96, 0.21, -0.44),
                           ("O2", (2.643, -0.722, 0.0), 3.0, 0.17, -0.53),
                           ("C2", (0.1, -0.78, 0.0), 3.5, 0.066, -0.12),
                           ("C3", (-1.06, 0.212, 0.0), 3.5, 0.066, -0.12),
                           ("C4", (-2.381, -0.551, 0.0), 3.5, 0.066, -0.18),
                           ("OH", (3.21, -0.461, 0.882), 3.4, 0.046, 0.45),
                           ("H2", (0.043, -1.407, 0.89), 2.5, 0.03, 0.06),
                           ("H3", (0.043, -1.407, -0.89), 2.5, 0.03, 0.06),
                           ("H4", (-1.002, 0.838, -0.89), 2.5, 0.03, 0.06),
                           ("H5", (-1.002, 0.838, 0.89), 2.5, 0.03, 0.06),
                           ("H6", (-2.439, -1.178, 0.89), 2.5, 0.03, 0.06),
                           ("H7", (-2.439, -1.178, -0.89), 2.5, 0.03, 0.06),
                           ("H8", (-3.21, 0.157, 0.0), 2.5, 0.03, 0.06)]),
    # guile/solutes.scm:438-458
    "hexane": _mol([("C", (1.709, -2.812, 0.0), 3.5, 0.066, -0.18),
                    ("C", (1.684, -1.278, 0.0), 3.5, 0.066, -0.12),
                    ("C", (0.245, -0.753, 0.0), 3.5, 0.066, -0.12),
                    ("C", (0.241, 0.779, 0.0), 3.5, 0.066, -0.12),
                    ("C", (-1.198, 1.304, 0.0), 3.5, 0.066, -0.12),
                    ("C", (-1.206, 2.834, 0.0), 3.5, 0.066, -0.18),
                    ("H", (2.236, -3.164, 0.887), 2.5, 0.03, 0.06),
                    ("H", (2.232, -3.164, -0.89), 2.5, 0.03, 0.06),
                    ("H", (0.691, -3.204, 0.003), 2.5, 0.03, 0.06),
                    ("H", (2.202, -0.914, -0.888), 2.5, 0.03, 0.06),
                    ("H", (2.201, -0.914, 0.89), 2.5, 0.03, 0.06),
                    ("H", (-0.273, -1.115, 0.889), 2.5, 0.03, 0.06),
                    ("H", (-0.272, -1.115, -0.89), 2.5, 0.03, 0.06),
                    ("H", (0.757, 1.142, -0.89), 2.5, 0.03, 0.06),
                    ("H", (0.757, 1.141, 0.89), 2.5, 0.03, 0.06),
                    ("H", (-1.716, 0.944, 0.89), 2.5, 0.03, 0.06),
                    ("H", (-1.716, 0.944, -0.89), 2.5, 0.03, 0.06),
                    ("H", (-0.696, 3.204, -0.89), 2.5, 0.03, 0.06),
                    ("H", (-0.696, 3.204, 0.89), 2.5, 0.03, 0.06),
                    ("H", (-2.236, 3.19, 0.0), 2.5, 0.03, 0.06)]),
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
