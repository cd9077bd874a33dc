"""ctypes binding of ``libpycfd_b200.so`` (the C ABI in ``include/pycfd_b200.h``).

The library is built in-tree by :mod:`pycfd_b200.build`.  Loading fails loudly
when it is missing: the package has no CPU fallback for the hot path.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpycfd_b200.so")

PCFD_E_ARG, PCFD_E_CUDA, PCFD_E_NOCONV, PCFD_E_STALL, PCFD_E_UNSUPPORTED = -1, -2, -3, -4, -5

BC_CODES = {"no_slip": 0, "moving_wall": 1, "inlet": 2, "outlet": 3, "pressure_outlet": 4,
            "periodic": 5, "symmetry": 6}
SOLVER_CODES = {"cg": 1, "jacobi": 2, "sor": 3, "multigrid": 4, "mgcg": 5}
SCHEME_CODES = {"euler": 0, "rk2": 1, "rk3": 2}
MAX_BODIES = 8

# Every exported symbol of the C ABI (checked against the header by the tests).
EXPORTS = (
    "pycfd_last_error", "pycfd_version", "pycfd_solver_create", "pycfd_solver_destroy",
    "pycfd_momentum_rhs", "pycfd_momentum_rhs_les", "pycfd_divergence", "pycfd_solver_momentum_rhs",
    "pycfd_solver_divergence", "pycfd_solver_momentum_rhs_les", "pycfd_apply_velocity_bc", "pycfd_poisson_solve",
    "pycfd_mg_apply", "pycfd_project", "pycfd_initialize", "pycfd_substep", "pycfd_step",
    "pycfd_step_graph", "pycfd_step_adaptive", "pycfd_set_clock", "pycfd_get_clock",
    "pycfd_history_read",
    "pycfd_step_host", "pycfd_get_stats", "pycfd_reduce_fields", "pycfd_face_lists", "pycfd_rasterize", "pycfd_adjoint_apply",
    "pycfd_reduce_fields_noalloc", "pycfd_profile_kernel", "pycfd_solver_persistent",
    "pycfd_solver_set_wait_limit", "pycfd_solve_trace", "pycfd_launch_count",
    "pycfd_profile_read", "pycfd_batch_create", "pycfd_batch_destroy", "pycfd_batch_initialize",
    "pycfd_batch_step", "pycfd_batch_problem", "pycfd_batch_status", "pycfd_batch_launches",
    "pycfd_batch_profile", "pycfd_batch_profile_read", "pycfd_batch_set_loop_cap",
    "pycfd_batch_capped",
)

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


class Shape(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_double * 4), ("verts", C.c_void_p), ("n_verts", C.c_int),
                ("image", C.c_void_p), ("rows", C.c_int), ("cols", C.c_int), ("threshold", C.c_double),
                ("invert", C.c_int)]


class AdjArgs(C.Structure):
    _fields_ = [("n", C.c_int), ("h", C.c_double), ("nu", C.c_double), ("dt", C.c_double),
                ("ca", C.c_double), ("cb", C.c_double), ("count", C.c_long),
                ("u", C.c_void_p), ("v", C.c_void_p), ("gu", C.c_void_p), ("gv", C.c_void_p),
                ("a", C.c_void_p), ("b", C.c_void_p), ("lid", C.c_void_p), ("cu", C.c_void_p),
                ("cv", C.c_void_p), ("lower", C.c_void_p), ("out_u", C.c_void_p), ("out_v", C.c_void_p),
                ("out", C.c_void_p), ("acc_u", C.c_void_p), ("acc_v", C.c_void_p)]


class MgLevel(C.Structure):
    _fields_ = [("n", C.c_int), ("shape_x", C.c_int), ("shape_y", C.c_int),
                ("weight", C.c_double), ("weighted_dinv", _dp), ("active", _u8p),
                ("a_indptr", C.POINTER(C.c_int64)), ("a_indices", C.POINTER(C.c_int32)),
                ("a_data", _dp), ("p_indptr", C.POINTER(C.c_int64)),
                ("p_indices", C.POINTER(C.c_int32)), ("p_data", _dp),
                ("m_indptr", C.POINTER(C.c_int64)), ("m_indices", C.POINTER(C.c_int32)),
                ("m_data", _dp)]


class SolverDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("nu", C.c_double), ("body_fx", C.c_double), ("body_fy", C.c_double),
                ("bc_kind", C.c_int * 4), ("bc_velocity", C.c_double * 4),
                ("bc_p_ref", C.c_double * 4), ("bc_profile", _dp * 4), ("solid", _u8p),
                ("body_id", _u8p), ("n_bodies", C.c_int), ("solver_kind", C.c_int),
                ("tol", C.c_double), ("maxiter", C.c_int), ("sor_omega", C.c_double),
                ("mg_sweeps", C.c_int), ("time_scheme", C.c_int), ("precision", C.c_int),
                ("inner_tol", C.c_double), ("n_levels", C.c_int),
                ("levels", C.POINTER(MgLevel)), ("coarsest_inverse", _dp),
                ("coarse_cluster_rows", C.c_int), ("sequential_launch", C.c_int),
                ("persistent_solve", C.c_int), ("tail_level", C.c_int), ("tail_operator", _dp),
                ("ell_thread_budget", C.c_int), ("use_les", C.c_int), ("les_coeff", C.c_double),
                ("metrics", C.POINTER(C.c_double)), ("outlet_width", C.c_double),
                ("les_coeff_field", C.POINTER(C.c_double))]


class DtControl(C.Structure):
    _fields_ = [("adaptive", C.c_int), ("cfl", C.c_double), ("visc_limit", C.c_double),
                ("dt_cap", C.c_double), ("t_end", C.c_double), ("blend_mode", C.c_int),
                ("blend", C.c_double), ("steady_tol", C.c_double), ("history", C.c_int)]


class BatchOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("tol", C.c_double), ("maxiter", C.c_int),
                ("inner_tol", C.c_double), ("mg_sweeps", C.c_int), ("tile_rows", C.c_int),
                ("coarse_level", C.c_int), ("fused_from", C.c_int), ("ell_group", C.c_int),
                ("programmatic_launch", C.c_int), ("stencil_transfer", C.c_int),
                ("scalar_strips", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("status", C.c_int),
                ("total_iterations", C.c_int), ("last_residual", C.c_double),
                ("fx", C.c_double), ("fy", C.c_double),
                ("body_fx", C.c_double * MAX_BODIES), ("body_fy", C.c_double * MAX_BODIES),
                ("ir_iterations", C.c_int), ("pad_", C.c_int)]


class FieldStats(C.Structure):
    _fields_ = [("max_u", C.c_double), ("max_v", C.c_double), ("max_du", C.c_double),
                ("max_dv", C.c_double), ("max_div", C.c_double),
                ("kinetic_energy", C.c_double), ("max_vorticity", C.c_double),
                ("finite", C.c_int), ("pad_", C.c_int)]


_lib = None


def load(path: str = LIB_PATH):
    """Load the library (once) and declare the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"pycfd_b200 native library not found at {path}; build it with "
            "`python -m pycfd_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    vp = C.c_void_p
    sig = {
        "pycfd_last_error": (C.c_char_p, []),
        "pycfd_version": (C.c_int, []),
        "pycfd_solver_create": (C.c_int, [C.POINTER(SolverDesc), C.POINTER(vp)]),
        "pycfd_solver_destroy": (C.c_int, [vp]),
        "pycfd_momentum_rhs": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_double, C.c_double,
                                         vp, vp, vp]),
        "pycfd_momentum_rhs_les": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                             C.c_double, C.c_double, C.c_double, C.c_double, vp, vp, vp, vp,
                                             vp]),
        "pycfd_divergence": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_double, C.c_double, vp, vp]),
        "pycfd_solver_momentum_rhs": (C.c_int, [vp, vp, vp, C.c_double, vp, vp, vp]),
        "pycfd_solver_divergence": (C.c_int, [vp, vp, vp, vp, vp]),
        "pycfd_solver_momentum_rhs_les": (C.c_int, [vp, vp, vp, C.c_double, vp, vp, vp, vp, vp]),
        "pycfd_apply_velocity_bc": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, vp]),
        "pycfd_poisson_solve": (C.c_int, [vp, vp, vp, vp, vp]),
        "pycfd_mg_apply": (C.c_int, [vp, vp, vp, vp]),
        "pycfd_project": (C.c_int, [vp, vp, vp, vp, C.c_double, vp]),
        "pycfd_initialize": (C.c_int, [vp, vp, vp, vp, vp]),
        "pycfd_substep": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, vp]),
        "pycfd_step": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, vp]),
        "pycfd_step_graph": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, vp]),
        "pycfd_step_host": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, vp]),
        "pycfd_step_adaptive": (C.c_int, [vp, vp, vp, vp, vp, vp, C.POINTER(DtControl), vp]),
        "pycfd_set_clock": (C.c_int, [vp, C.c_double, vp]),
        "pycfd_history_read": (C.c_int, [vp, vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), vp]),
        "pycfd_get_clock": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_int), C.POINTER(C.c_int), vp]),
        "pycfd_get_stats": (C.c_int, [vp, C.POINTER(Stats), vp]),
        "pycfd_profile_kernel": (C.c_int, [vp, C.c_int]),
        "pycfd_solver_persistent": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "pycfd_solver_set_wait_limit": (C.c_int, [vp, C.c_ulonglong]),
        "pycfd_solve_trace": (C.c_int, [vp, C.c_int, C.POINTER(C.c_ulonglong), C.c_int, vp]),
        "pycfd_launch_count": (C.c_longlong, []),
        "pycfd_profile_read": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int), vp]),
        "pycfd_reduce_fields": (C.c_int, [vp, vp, vp, vp, vp, vp, C.POINTER(FieldStats), vp]),
        "pycfd_adjoint_apply": (C.c_int, [C.c_int, C.POINTER(AdjArgs), vp]),
        "pycfd_rasterize": (C.c_int, [C.POINTER(Shape), vp, vp, vp, vp, C.c_int, C.c_int, C.c_double,
                                      C.c_double, C.c_int, vp, vp, vp]),
        "pycfd_face_lists": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), vp, vp, C.POINTER(C.c_int), vp]),
        "pycfd_reduce_fields_noalloc": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_int, C.c_int,
                                                  C.c_double, C.c_double, C.POINTER(FieldStats),
                                                  vp]),
        "pycfd_batch_create": (C.c_int, [C.POINTER(SolverDesc), C.POINTER(C.c_int),
                                         C.POINTER(DtControl), C.POINTER(C.c_int), C.POINTER(vp),
                                         C.POINTER(vp), C.POINTER(vp), C.c_int,
                                         C.POINTER(BatchOpts), C.POINTER(vp)]),
        "pycfd_batch_destroy": (C.c_int, [vp]),
        "pycfd_batch_initialize": (C.c_int, [vp, vp]),
        "pycfd_batch_step": (C.c_int, [vp, C.c_int, C.c_int, vp]),
        "pycfd_batch_problem": (vp, [vp, C.c_int]),
        "pycfd_batch_status": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), vp]),
        "pycfd_batch_launches": (C.c_int, [vp, C.c_int, C.POINTER(C.c_longlong), vp]),
        "pycfd_batch_profile": (C.c_int, [vp, C.c_int]),
        "pycfd_batch_set_loop_cap": (C.c_int, [vp, C.c_int, vp]),
        "pycfd_batch_capped": (C.c_int, [vp, C.POINTER(C.c_int), vp]),
        "pycfd_batch_profile_read": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int), vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class NativeError(RuntimeError):
    """A CUDA runtime failure inside the native library."""


def check(rc: int) -> None:
    """Map a status code onto the reference's exception types."""
    if rc == 0:
        return
    msg = _lib.pycfd_last_error().decode() if _lib is not None else ""
    if rc == PCFD_E_ARG:
        raise ValueError(msg)
    if rc == PCFD_E_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc in (PCFD_E_NOCONV, PCFD_E_STALL):
        raise RuntimeError(msg)
    raise NativeError(msg or f"native call failed with status {rc}")


def ptr(t) -> C.c_void_p:
    """Device (or host) address of a torch tensor / numpy array / None."""
    if t is None:
        return C.c_void_p(0)
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return C.c_void_p(t.ctypes.data)


def cast(a, ctype):
    """numpy array -> typed ctypes pointer (None -> NULL)."""
    if a is None:
        return C.cast(C.c_void_p(0), C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))
