"""ctypes binding of libjxb.so (the C ABI declared in include/jxb.h).

The shared library is built in-tree (``jaxiga_b200/libjxb.so``) by
``jaxiga_b200/build.py``. Loading it needs no GPU; every compute call does.
There is no CPU fallback: when the library is missing, importing the solver
path raises.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libjxb.so")

OP_POISSON, OP_ELASTICITY, OP_PLATE, OP_HYPERELASTIC = 0, 1, 2, 3

STATUS = {0: "OK", 1: "invalid argument", 2: "CUDA error", 3: "not converged", 4: "non-finite", 5: "out of memory"}

c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_int32_p = ctypes.POINTER(ctypes.c_int32)


class Desc(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("vec", ctypes.c_int),
        ("degree", ctypes.c_int),
        ("n_quad", ctypes.c_int),
        ("n_cp", ctypes.c_int * 3),
        ("n_span", ctypes.c_int * 3),
        ("first", c_int32_p * 3),
        ("span_lo", c_double_p * 3),
        ("span_hi", c_double_p * 3),
        ("extraction", c_double_p * 3),
        ("cpts", c_double_p),
        ("wgts", c_double_p),
        ("gauss_nodes", c_double_p),
        ("gauss_weights", c_double_p),
        ("op", ctypes.c_int),
        ("coef", ctypes.c_double * 4),
        ("plane_strain", ctypes.c_int),
        ("coef_qp", c_double_p),
        ("prescribed", ctypes.POINTER(ctypes.c_uint8)),
        ("want_f32", ctypes.c_int),
        ("tile", ctypes.c_int * 2),
    ]


class ThbDesc(ctypes.Structure):
    """jxb_thb_desc (include/jxb.h)."""

    _fields_ = [
        ("dim", ctypes.c_int),
        ("degree", ctypes.c_int),
        ("n_local_max", ctypes.c_int),
        ("op", ctypes.c_int),
        ("n_elem", ctypes.c_int64),
        ("n_scalar", ctypes.c_int64),
        ("lam", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("elem_dofs", ctypes.c_void_p),
        ("extraction", ctypes.c_void_p),
        ("wgts", ctypes.c_void_p),
        ("tables", ctypes.c_void_p),
        ("factors", ctypes.c_void_p),
        ("wq", ctypes.c_void_p),
        ("prescribed", ctypes.c_void_p),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("n_dofs", ctypes.c_int64),
        ("n_free", ctypes.c_int64),
        ("n_elem", ctypes.c_int64),
        ("n_qp", ctypes.c_int64),
        ("n_bricks", ctypes.c_int64),
        ("geo_bytes", ctypes.c_int64),
        ("scratch_bytes", ctypes.c_int64),
        ("ngeo", ctypes.c_int),
        ("rational", ctypes.c_int),
    ]


class SolveOpts(ctypes.Structure):
    _fields_ = [
        ("tol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("maxiter", ctypes.c_int64),
        ("preconditioner", ctypes.c_int),
        ("check_every", ctypes.c_int),
        ("inner_tol", ctypes.c_double),
        ("max_outer", ctypes.c_int),
        ("restarts", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int64),
        ("outer", ctypes.c_int64),
        ("residual", ctypes.c_double),
        ("relative_residual", ctypes.c_double),
        ("b_norm", ctypes.c_double),
        ("converged", ctypes.c_int),
        ("finite", ctypes.c_int),
        ("seconds", ctypes.c_double),
    ]


class Transfer1d(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_int),
        ("cols", ctypes.c_int),
        ("ptr", c_int32_p),
        ("idx", c_int32_p),
        ("val", c_double_p),
    ]


# (name, argtypes) of every exported entry point, in include/jxb.h order
SIGNATURES = [
    ("jxb_plan_create", [ctypes.POINTER(Desc), ctypes.POINTER(ctypes.c_void_p)]),
    ("jxb_plan_destroy", [ctypes.c_void_p]),
    ("jxb_plan_info", [ctypes.c_void_p, ctypes.POINTER(Info)]),
    ("jxb_last_error", []),
    ("jxb_version", []),
    ("jxb_apply", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    ("jxb_apply_f32", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_apply_static", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    ("jxb_diag", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_qp_coords", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_interpolate", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("jxb_interpolate_grad", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("jxb_boundary_points", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_void_p]),
    ("jxb_boundary_load", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_eval_points", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                         ctypes.c_void_p]),
    ("jxb_load", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_qp_weights", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_pcg", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                 ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    ("jxb_refine_solve", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                          ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    ("jxb_mixed_pcg", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    ("jxb_bicgstab", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                      ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    ("jxb_pcg_snapshots", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.POINTER(SolveOpts), ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                           c_int64_p, ctypes.POINTER(Stats)]),
    ("jxb_batch_create", [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("jxb_batch_destroy", [ctypes.c_void_p]),
    ("jxb_mp_create", [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                       ctypes.POINTER(ctypes.c_void_p)]),
    ("jxb_thb_create", [ctypes.POINTER(ThbDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ("jxb_hyper_state", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ("jxb_hyper_residual", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_batch_size", [ctypes.c_void_p, c_int64_p, c_int64_p]),
    ("jxb_batch_info", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("jxb_batch_apply", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_batch_pcg", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats), c_double_p]),
    ("jxb_cnn_create", [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int32_p, ctypes.c_uint64,
                        ctypes.POINTER(ctypes.c_void_p)]),
    ("jxb_cnn_destroy", [ctypes.c_void_p]),
    ("jxb_cnn_set_input_pooling", [ctypes.c_void_p, ctypes.c_int]),
    ("jxb_cnn_set_inference_bf16", [ctypes.c_void_p, ctypes.c_int]),
    ("jxb_cnn_params", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), c_int64_p]),
    ("jxb_cnn_grads", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), c_int64_p]),
    ("jxb_cnn_forward", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                         ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_cnn_backward", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_cnn_zero_grad", [ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_cnn_accumulate", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, c_double_p]),
    ("jxb_cnn_accumulate_energy", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_double, ctypes.c_int,
                                   c_double_p]),
    ("jxb_cnn_adam", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_float]),
    ("jxb_fcg_learned", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                         ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_int,
                         ctypes.c_int, ctypes.c_int, ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    ("jxb_mg_create", [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(Transfer1d), c_double_p,
                       ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]),
    ("jxb_mg_destroy", [ctypes.c_void_p]),
    ("jxb_mg_info", [ctypes.c_void_p, c_double_p]),
    ("jxb_mg_vcycle", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_mg_pcg", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                    ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    ("jxb_csr_create", [ctypes.c_int64, c_int64_p, c_int32_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("jxb_csr_destroy", [ctypes.c_void_p]),
    ("jxb_csr_matvec", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("jxb_csr_pcg", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                     ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    ("jxb_dot", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, c_double_p]),
    ("jxb_profile_apply", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                           ctypes.c_int, c_double_p]),
]

_lib = None


def load():
    """Load libjxb.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libjxb.so not found at {LIB_PATH}; build it with `python -m jaxiga_b200.build` "
            "(the B200 solver has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_char_p if name == "jxb_last_error" else ctypes.c_int
    _lib = lib
    return lib


class JxbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libjxb error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


def check(code):
    if code != 0:
        msg = load().jxb_last_error()
        raise JxbError(code, msg.decode() if msg else "")
    return code


NOT_CONVERGED, NONFINITE = 3, 4


def check_solve(code, raise_on_nonfinite=False):
    """Status of a solve entry point. The solves write x and the stats before
    returning JXB_ERR_NOT_CONVERGED or JXB_ERR_NONFINITE; both are reported
    through the stats (the reference's diagnostics report a failed solve the
    same way), so only the other codes raise, and NONFINITE when asked."""
    if code == NOT_CONVERGED or (code == NONFINITE and not raise_on_nonfinite):
        return code
    return check(code)
