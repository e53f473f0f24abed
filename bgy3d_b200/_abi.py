"""ctypes binding of include/rism3d.h (librism3d.so, built in-tree).

The library is the product: there is no Python or CPU fallback.  Importing
this module raises if the shared object is missing.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librism3d.so")

# Enumerations (rism3d.h)
HNC, KH, PY = 0, 1, 2
PSE0 = 3
CLOSURES = {"HNC": 0, "KH": 1, "PY": 2, **{f"PSE{n}": 3 + n for n in range(8)}}
NEWTON, PICARD, TRIAL, JAGER = 0, 1, 2, 3
SOLVERS = {"newton": NEWTON, "picard": PICARD, "trial": TRIAL, "jager": JAGER}
FP64, MIXED = 0, 1

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_TABLE, ERR_NOT_CONVERGED, ERR_NAN, ERR_UNSUPPORTED = range(-1, -8, -1)
ERRORS = {
    -1: "bad argument", -2: "CUDA error", -3: "out of device memory",
    -4: "|k| beyond the chi table", -5: "not converged", -6: "NaN residual",
    -7: "unsupported",
}


class Site(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 8), ("x", ctypes.c_double * 3),
                ("sigma", ctypes.c_double), ("epsilon", ctypes.c_double),
                ("charge", ctypes.c_double)]


class Problem(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int * 3), ("L", ctypes.c_double * 3),
                ("beta", ctypes.c_double), ("rho", ctypes.c_double),
                ("rmax", ctypes.c_double), ("nrad", ctypes.c_int),
                ("closure", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("norm_tol", ctypes.c_double), ("lambda_", ctypes.c_double),
                ("solver", ctypes.c_int), ("renorm", ctypes.c_int),
                ("precision", ctypes.c_int), ("verbosity", ctypes.c_int),
                ("krylov_restart", ctypes.c_int), ("ew_forcing", ctypes.c_int),
                ("coarse_h", ctypes.c_double), ("coarse_steps", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("mu", ctypes.c_double), ("mu_hnc", ctypes.c_double),
                ("mu_kh", ctypes.c_double), ("mu_gf", ctypes.c_double),
                ("pmv_factor", ctypes.c_double), ("resid_inf", ctypes.c_double),
                ("resid_2", ctypes.c_double), ("status", ctypes.c_int),
                ("newton_iters", ctypes.c_int), ("f_evals", ctypes.c_int),
                ("jv_evals", ctypes.c_int), ("f_evals_fp32", ctypes.c_int),
                ("jv_evals_fp32", ctypes.c_int), ("jv_evals_coarse", ctypes.c_int),
                ("seconds", ctypes.c_double), ("launches", ctypes.c_longlong)]


class Job(ctypes.Structure):
    _fields_ = [("pd", Problem), ("n", ctypes.c_int), ("solute", ctypes.POINTER(Site)),
                ("chi", ctypes.POINTER(ctypes.c_double)), ("t_inout", ctypes.POINTER(ctypes.c_double)),
                ("g_out", ctypes.POINTER(ctypes.c_double)), ("result", Result)]


class Grad(ctypes.Structure):
    _fields_ = [("dq", ctypes.POINTER(ctypes.c_double)), ("dsigma", ctypes.POINTER(ctypes.c_double)),
                ("depsilon", ctypes.POINTER(ctypes.c_double)), ("dx", ctypes.POINTER(ctypes.c_double)),
                ("adjoint_jv", ctypes.c_int), ("adjoint_resid", ctypes.c_double), ("seconds", ctypes.c_double),
                ("dx_reference", ctypes.POINTER(ctypes.c_double))]


class SolventResult(ctypes.Structure):
    _fields_ = [("mu", ctypes.c_double), ("mu_hnc", ctypes.c_double), ("mu_kh", ctypes.c_double),
                ("mu_gf", ctypes.c_double), ("a", ctypes.c_double), ("kappa", ctypes.c_double),
                ("resid_inf", ctypes.c_double), ("resid_2", ctypes.c_double), ("status", ctypes.c_int),
                ("newton_iters", ctypes.c_int), ("f_evals", ctypes.c_int), ("jv_evals", ctypes.c_int),
                ("seconds", ctypes.c_double)]


D3 = ctypes.c_double * 3
D33 = (ctypes.c_double * 3) * 3


class InfoResult(ctypes.Structure):
    _fields_ = [("q_u", ctypes.c_double), ("d_u", D3), ("Q_u", D33), ("q_v", ctypes.c_double), ("d_v", D3),
                ("Q_v", D33), ("d_n", D3), ("U_v_rho_N", ctypes.c_double), ("U_v_rho_N_trilinear", ctypes.c_double),
                ("U_v_rho_u", ctypes.c_double), ("rho_v_U_u", ctypes.c_double), ("seconds", ctypes.c_double)]


# Every entry point declared in include/rism3d.h (checked by the CPU tests).
EXPORTS = [
    "rism3d_problem_defaults", "rism3d_solute_solve", "rism3d_ctx_create",
    "rism3d_ctx_destroy", "rism3d_ctx_size", "rism3d_iterate_t1",
    "rism3d_jacobian_t1", "rism3d_iterate_t1_f32", "rism3d_jacobian_t1_f32",
    "rism3d_solve", "rism3d_observables", "rism3d_get_field", "rism3d_last_error",
    "rism3d_profile", "rism1d_solvent_chi", "rism3d_jacobian_apply_noalloc",
    "rism3d_precondition", "rism3d_precondition_f32", "rism3d_coarse_grid", "rism3d_coarse_driver", "rism3d_solve_batch",
    "rism3d_solute_grad", "rism3d_gradient", "rism3d_jacobian_transpose_t1", "rism3d_ctx_set_solute",
    "rism3d_response", "rism3d_solvent_solve", "rism3d_solvent_ctx_create", "rism3d_ctx_create_chi3",
    "rism3d_solute_solve_chi3", "rism3d_info", "rism3d_moments", "rism3d_tile_shapes",
    "rism3d_free_energy_gradient", "rism3d_cache_clear",
]

_lib = None


def lib():
    """Load librism3d.so once; raise if it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m bgy3d_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P, I, D, V = ctypes.POINTER, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    L.rism3d_problem_defaults.argtypes = [P(Problem), D, I]
    L.rism3d_problem_defaults.restype = None
    L.rism3d_solute_solve.argtypes = [P(Problem), I, P(Site), I, P(Site), P(D), P(D), P(D), P(Result)]
    L.rism3d_solute_solve.restype = I
    L.rism3d_ctx_create.argtypes = [P(Problem), I, P(Site), I, P(Site), P(D), P(V)]
    L.rism3d_ctx_create.restype = I
    L.rism3d_ctx_destroy.argtypes = [V]
    L.rism3d_ctx_destroy.restype = None
    L.rism3d_ctx_size.argtypes = [V]
    L.rism3d_ctx_size.restype = ctypes.c_longlong
    for name in ("rism3d_iterate_t1", "rism3d_iterate_t1_f32"):
        getattr(L, name).argtypes = [V, V, V, P(D)]
        getattr(L, name).restype = I
    for name in ("rism3d_jacobian_t1", "rism3d_jacobian_t1_f32"):
        getattr(L, name).argtypes = [V, V, V, V]
        getattr(L, name).restype = I
    L.rism3d_solve.argtypes = [V, V, P(Result)]
    L.rism3d_solve.restype = I
    L.rism3d_observables.argtypes = [V, V, V, P(Result)]
    L.rism3d_observables.restype = I
    L.rism3d_get_field.argtypes = [V, I, V]
    L.rism3d_get_field.restype = I
    L.rism3d_last_error.argtypes = []
    L.rism3d_last_error.restype = ctypes.c_char_p
    L.rism3d_profile.argtypes = [V, I, P(D), P(ctypes.c_longlong)]
    L.rism3d_profile.restype = I
    L.rism1d_solvent_chi.argtypes = [P(Problem), D, I, P(Site), P(D), P(D), P(D)]
    L.rism1d_solvent_chi.restype = I
    L.rism3d_jacobian_apply_noalloc.argtypes = [P(Problem), I, P(D), V, V, V]
    L.rism3d_jacobian_apply_noalloc.restype = I
    L.rism3d_precondition.argtypes = [V, V, V, V]
    L.rism3d_precondition.restype = I
    L.rism3d_precondition_f32.argtypes = [V, V, V, V]
    L.rism3d_precondition_f32.restype = I
    L.rism3d_coarse_grid.argtypes = [V, P(I)]
    L.rism3d_coarse_grid.restype = I
    L.rism3d_coarse_driver.argtypes = [V]
    L.rism3d_coarse_driver.restype = I
    L.rism3d_cache_clear.argtypes = []
    L.rism3d_cache_clear.restype = None
    L.rism3d_solve_batch.argtypes = [I, P(Site), I, P(Job), I]
    L.rism3d_solve_batch.restype = I
    L.rism3d_solute_grad.argtypes = [P(Problem), I, P(Site), I, P(Site), P(D), P(D), P(Result), P(Grad)]
    L.rism3d_solute_grad.restype = I
    L.rism3d_gradient.argtypes = [V, V, P(Grad)]
    L.rism3d_gradient.restype = I
    L.rism3d_jacobian_transpose_t1.argtypes = [V, V, V, V]
    L.rism3d_jacobian_transpose_t1.restype = I
    L.rism3d_ctx_set_solute.argtypes = [V, I, P(Site)]
    L.rism3d_ctx_set_solute.restype = I
    L.rism3d_response.argtypes = [V, V, P(Grad)]
    L.rism3d_response.restype = I
    L.rism3d_solvent_solve.argtypes = [P(Problem), I, P(Site), P(D), P(D), P(D), P(D), P(SolventResult)]
    L.rism3d_solvent_solve.restype = I
    L.rism3d_solvent_ctx_create.argtypes = [P(Problem), I, P(Site), P(V)]
    L.rism3d_solvent_ctx_create.restype = I
    L.rism3d_ctx_create_chi3.argtypes = [P(Problem), I, P(Site), I, P(Site), P(D), P(V)]
    L.rism3d_ctx_create_chi3.restype = I
    L.rism3d_solute_solve_chi3.argtypes = [P(Problem), I, P(Site), I, P(Site), P(D), P(D), P(D), P(Result)]
    L.rism3d_solute_solve_chi3.restype = I
    L.rism3d_info.argtypes = [V, V, P(InfoResult), P(D)]
    L.rism3d_info.restype = I
    L.rism3d_moments.argtypes = [V, V, I, P(D)]
    L.rism3d_moments.restype = I
    L.rism3d_tile_shapes.argtypes = [V, P(I)]
    L.rism3d_tile_shapes.restype = I
    L.rism3d_free_energy_gradient.argtypes = [V, V, P(D)]
    L.rism3d_free_energy_gradient.restype = I
    _lib = L
    return L


class RismError(RuntimeError):
    def __init__(self, code, where=""):
        msg = ERRORS.get(code, f"error {code}")
        detail = lib().rism3d_last_error().decode(errors="replace") if _lib else ""
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail else ""))
        self.code = code


def check(code, where):
    if code != OK:
        raise RismError(code, where)
    return code
