"""Loader and ctypes signatures of libyafel_b200.so (the C ABI of include/yafel_gpu.h).

There is no fallback: if the library is missing it is built with nvcc, and if
that fails the import fails.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libyafel_b200.so")
_LIB = None

YG_OK, YG_NOT_CONVERGED, YG_BREAKDOWN, YG_NAN, YG_TIMEOUT, YG_OUT_OF_MEMORY, YG_OVER_BUDGET, \
    YG_BAD_ARG, YG_CUDA_ERROR, YG_UNSUPPORTED, YG_ZERO_PIVOT, YG_RUNNING = range(12)

vp = C.c_void_p
i32, i64, u32, u64, f64 = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_double
P = C.POINTER


class Physics(C.Structure):
    _fields_ = [("kind", i32), ("nsd", i32), ("params", f64 * 8)]


class SolveOpts(C.Structure):
    _fields_ = [("criterion", i32), ("precision", i32), ("tol", f64), ("maxiter", i64),
                ("check_every", i32), ("profile", i32)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", i64), ("rel_residual", f64), ("status", i32), ("refinements", i32),
                ("device_ms", f64), ("spmv_ms", f64), ("spmv_launches", i64)]


# name -> (restype, argtypes); mirrors include/yafel_gpu.h
SIGNATURES = {
    "yg_context_create": (i32, [i32, u64, P(vp)]),
    "yg_context_destroy": (i32, [vp]),
    "yg_context_synchronize": (i32, [vp]),
    "yg_context_memory": (i32, [vp, P(u64), P(u64)]),
    "yg_context_launches": (i64, [vp]),
    "yg_last_error": (C.c_char_p, []),
    "yg_status_string": (C.c_char_p, [i32]),
    "yg_vector_create": (i32, [vp, i64, P(vp)]),
    "yg_vector_destroy": (i32, [vp]),
    "yg_vector_size": (i64, [vp]),
    "yg_vector_upload": (i32, [vp, vp, i64]),
    "yg_vector_download": (i32, [vp, vp, i64]),
    "yg_vector_fill": (i32, [vp, f64]),
    "yg_vector_copy": (i32, [vp, vp]),
    "yg_vector_dot": (i32, [vp, vp, P(f64)]),
    "yg_vector_axpy": (i32, [f64, vp, vp]),
    "yg_dofmap_create": (i32, [vp, vp, i32, vp, vp, vp, i32, i32, i32, P(vp)]),
    "yg_dofmap_destroy": (i32, [vp]),
    "yg_dofmap_create_on_device": (i32, [vp, vp, i32, vp, vp, vp, i32, i32, i32, P(vp)]),
    "yg_dofmap_create_box": (i32, [vp, i32, i32, i32, i32, f64, f64, f64, i32, i32, P(vp)]),
    "yg_dofmap_sizes": (i32, [vp, P(i32), P(i32), P(i64), P(i64)]),
    "yg_dofmap_get": (i32, [vp, vp, vp, vp, vp, vp, vp]),
    "yg_dofmap_create_from_numbering": (i32, [vp, vp, i32, vp, vp, vp, i32, i32, i32, P(vp)]),
    "yg_element_table": (i32, [i32, i32, i32, P(i32), P(i32), vp, vp, vp, vp, vp]),
    "yg_zz_gradient_recovery": (i32, [vp, i32, vp, vp]),
    "yg_output_vtu": (i32, [vp, C.c_char_p, vp]),
    "yg_mesh_read_gmsh": (i32, [C.c_char_p, P(vp)]),
    "yg_mesh_sizes": (i32, [vp, P(i32), P(i32), P(i64), P(i64)]),
    "yg_mesh_get": (i32, [vp, vp, vp, vp, vp, vp, vp]),
    "yg_mesh_destroy": (i32, [vp]),
    "yg_assemble": (i32, [vp, P(Physics), u32, i32, P(vp), vp]),
    "yg_dirichlet_apply": (i32, [vp, vp, vp, vp, i64]),
    "yg_matrix_from_triplets": (i32, [vp, i32, vp, vp, vp, u64, P(vp)]),
    "yg_matrix_from_csr": (i32, [vp, i32, i64, i64, vp, vp, vp, P(vp)]),
    "yg_matrix_destroy": (i32, [vp]),
    "yg_matrix_sizes": (i32, [vp, P(i64), P(i64), P(i64), P(i32)]),
    "yg_matrix_get": (i32, [vp, vp, vp, vp]),
    "yg_matrix_make_fp32": (i32, [vp]),
    "yg_spmv": (i32, [vp, vp, vp]),
    "yg_spmv_ex": (i32, [vp, vp, vp, i32]),
    "yg_matrix_set_spmv": (i32, [vp, i32, i32]),
    "yg_matrix_set_spmv_for": (i32, [vp, i32, i32, i32]),
    "yg_matrix_get_spmv": (i32, [vp, P(i32), P(i32)]),
    "yg_matrix_get_spmv_for": (i32, [vp, i32, P(i32), P(i32)]),
    "yg_spmv_bench": (i32, [vp, vp, vp, i32, i32, P(f64)]),
    "yg_precond_create": (i32, [vp, i32, P(vp)]),
    "yg_precond_apply": (i32, [vp, vp]),
    "yg_precond_destroy": (i32, [vp]),
    "yg_precond_zero_pivots": (i64, [vp]),
    "yg_precond_levels": (i32, [vp, P(i64), P(i64)]),
    "yg_cg": (i32, [vp, vp, vp, vp, P(SolveOpts), P(SolveStats)]),
    "yg_bicgstab": (i32, [vp, vp, vp, vp, P(SolveOpts), P(SolveStats)]),
    "yg_batch_create": (i32, [vp, i32, P(vp)]),
    "yg_batch_destroy": (i32, [vp]),
    "yg_batch_add": (i32, [vp, vp, vp, vp, i32, P(SolveOpts), P(i32)]),
    "yg_batch_work_bytes": (i64, [i64, i32]),
    "yg_batch_launch": (i32, [vp]),
    "yg_batch_wait": (i32, [vp, P(i32)]),
    "yg_batch_ready": (i32, [vp, P(i32)]),
    "yg_local_smoothing_gradient": (i32, [vp, i32, vp, vp]),
    "yg_batch_set_solo_bytes": (i32, [vp, i64]),
    "yg_batch_get_tuning": (i32, [vp, P(i32)]),
    "yg_batch_set_tuning": (i32, [vp, i32, i32, i32, i32]),
    "yg_server_create": (i32, [vp, u64, i32, P(vp)]),
    "yg_server_destroy": (i32, [vp]),
    "yg_server_submit": (i32, [vp, u64, P(i64)]),
    "yg_server_admit": (i32, [vp, P(i64)]),
    "yg_server_attach": (i32, [vp, i64, vp, vp, vp, i32, P(SolveOpts)]),
    "yg_server_launch": (i32, [vp]),
    "yg_server_wait": (i32, [vp, P(i32)]),
    "yg_server_ready": (i32, [vp, P(i32)]),
    "yg_server_set_solo_spmv_bytes": (i32, [vp, i64]),
    "yg_server_finished": (i32, [vp, P(i64), i32, P(i32)]),
    "yg_server_poll": (i32, [vp, i64, P(SolveStats)]),
    "yg_server_release": (i32, [vp, i64]),
    "yg_server_info": (i32, [vp, P(i64), P(i64), P(u64)]),
    "yg_server_tune": (i32, [vp]),
    "yg_server_set_solo_rows": (i32, [vp, i64]),
    "yg_batch_remove": (i32, [vp, i32]),
    "yg_batch_reset": (i32, [vp, i32]),
    "yg_batch_run": (i32, [vp, i32, P(i32)]),
    "yg_batch_stats": (i32, [vp, i32, P(SolveStats)]),
    "yg_batch_tune": (i32, [vp]),
    "yg_dot_static_scratch": (i32, [vp, vp, i64, vp, vp]),
}


class YafelError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d)" % (msg, status))
        self.status = status


def lib():
    """Load (building first if absent) libyafel_b200.so."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status, what=""):
    if status != YG_OK:
        msg = lib().yg_last_error().decode(errors="replace")
        raise YafelError(status, "%s: %s" % (what, msg) if what else msg)
    return status
