"""ctypes binding of libnnkifmm.so (declarations in include/nnkifmm.h).

The library is loaded from this directory only; there is no other
implementation.  If it is missing the import fails with the build command.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnnkifmm.so")

NNK_OK = 0
NNK_E_ARG = 1
NNK_E_MAXDEPTH = 2
NNK_E_NONFINITE = 3
NNK_E_NOCONV = 4
NNK_E_OOM = 5
NNK_E_CUDA = 6
NNK_E_TIMEOUT = 7
NNK_E_STATE = 8
LAYOUT_ROWS = 1
LAYOUT_BLOCKED = 2
PREC_FP64 = 0
PREC_MIXED = 1
PREC_NEAR32 = 2
NOALLOC_MAX_FINE = 262144
PHASES = ["gather", "up_pairs", "up_c2e", "down_pairs", "down_c2e", "leaf_pairs", "scatter", "m2l"]

_i32, _i64, _f64, _vp = C.c_int32, C.c_int64, C.c_double, C.c_void_p
_pd, _pi32, _pi64, _pu8 = (C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                           C.POINTER(C.c_uint8))


class TreeParams(C.Structure):
    _fields_ = [("node_capacity", _i32), ("max_depth", _i32), ("nearest", _i32), ("builder", _i32)]


class TreeInfo(C.Structure):
    _fields_ = [("num_points", _i64), ("num_potentials", _i64), ("num_targets", _i64), ("num_fine", _i64),
                ("nn_nnz", _i64), ("source_entries", _i64), ("u_total", _i64), ("v_total", _i64),
                ("w_total", _i64), ("x_total", _i64), ("node_count", _i32), ("max_level", _i32),
                ("node_capacity", _i32), ("nearest", _i32)]


class FmmParams(C.Structure):
    _fields_ = [("eps", _f64), ("mu", _f64), ("corona_res", _i32), ("corona_shells", _i32),
                ("precision", _i32), ("m2l_mode", _i32), ("reg", _f64)]


class FmmStats(C.Structure):
    _fields_ = [("pairs_leaf", _i64), ("pairs_p2p", _i64), ("pairs_up", _i64), ("pairs_down", _i64),
                ("m2l_pairs", _i64), ("c2e_columns", _i64), ("m2l_tile_rows", _i64), ("surface_points", _i32),
                ("levels", _i32), ("m2l_rank", _i32), ("folded", _i32), ("m2l_frequencies", _i32),
                ("m2l_family", _i32), ("m2l_records", _i64), ("m2l_groups", _i64), ("m2m_product_pairs", _i64),
                ("l2l_product_pairs", _i64)]


class SolveParams(C.Structure):
    _fields_ = [("tol", _f64), ("maxit", _i32), ("restart", _i32)]


class SolveInfo(C.Structure):
    _fields_ = [("flag", _i32), ("iters", _i32), ("relres", _f64)]


# name -> (restype, argtypes); every symbol declared in include/nnkifmm.h
SIGNATURES = {
    "nnk_version": (C.c_char_p, []),
    "nnk_ctx_create": (_i32, [_i32, C.POINTER(_vp)]),
    "nnk_ctx_destroy": (_i32, [_vp]),
    "nnk_ctx_set_stream": (_i32, [_vp, _vp]),
    "nnk_ctx_synchronize": (_i32, [_vp]),
    "nnk_last_error": (C.c_char_p, [_vp]),
    "nnk_nearest_matrix": (_i32, [_vp, _vp, _i64, _vp, _i64, _pi64, _vp, _vp, _vp]),
    "nnk_nearest_matrix_host": (_i32, [_vp, _vp, _i64, _vp, _i64, _pi64, _vp, _vp, _vp]),
    "nnk_nearest_reference_weights": (_i32, [_vp, _i64, _vp, _vp, _vp, _f64]),
    "nnk_tree_build": (_i32, [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _vp, C.POINTER(TreeParams),
                              C.POINTER(_vp)]),
    "nnk_tree_info_get": (_i32, [_vp, C.POINTER(TreeInfo)]),
    "nnk_tree_export_nodes": (_i32, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "nnk_tree_export_points": (_i32, [_vp, _vp, _vp, _vp]),
    "nnk_tree_export_list": (_i32, [_vp, _i32, _vp, _vp]),
    "nnk_tree_destroy": (_i32, [_vp]),
    "nnk_fmm_create": (_i32, [_vp, _vp, C.POINTER(FmmParams), C.POINTER(_vp)]),
    "nnk_fmm_apply": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32]),
    "nnk_fmm_apply_sparse": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32]),
    "nnk_fmm_reduced_apply": (_i32, [_vp, _vp, _vp, _i32, _i32]),
    "nnk_fmm_reduced_solve": (_i32, [_vp, _vp, _vp, _i32, _i32]),
    "nnk_fmm_stats_get": (_i32, [_vp, C.POINTER(FmmStats)]),
    "nnk_fmm_set_fold": (_i32, [_vp, _i32]),
    "nnk_fmm_set_c2e": (_i32, [_vp, _i32]),
    "nnk_fmm_set_m2m_form": (_i32, [_vp, _i32]),
    "nnk_measure_l2_read": (_i32, [_vp, C.POINTER(_f64)]),
    "nnk_fmm_c2e_mode": (_i32, [_vp, C.POINTER(_i32)]),
    "nnk_fmm_setup_times": (_i32, [_vp, C.POINTER(C.c_double), _i32]),
    "nnk_fmm_destroy": (_i32, [_vp]),
    "nnk_fmm_apply_adjoint": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32]),
    "nnk_fmm_source_count": (_i32, [_vp, _pi64]),
    "nnk_fmm_set_eps": (_i32, [_vp, _f64]),
    "nnk_fmm_autotune": (_i32, [_vp, _i32, _pd, _pd]),
    "nnk_fmm_grad_positions": (_i32, [_vp, _vp, _vp, _i32, _vp, _vp, _i32]),
    "nnk_fmm_grad_eps": (_i32, [_vp, _vp, _vp, _i32, _pd, _i32]),
    "nnk_fmm_profile": (_i32, [_vp, _i32]),
    "nnk_fmm_profile_read": (_i32, [_vp, _vp, _vp]),
    "nnk_fmm_test_wait_timeout": (_i32, [_vp, C.c_uint32]),
    "nnk_fmm_solve": (_i32, [_vp, _vp, _vp, _i32, C.POINTER(SolveParams), C.POINTER(SolveInfo), _i32]),
    "nnk_mob_create": (_i32, [_vp, _i32, _vp, _vp, _vp, _vp, C.POINTER(_vp)]),
    "nnk_mob_apply": (_i32, [_vp, _vp, _vp, _i32]),
    "nnk_mob_precon": (_i32, [_vp, _vp, _vp, _i32]),
    "nnk_mob_use_graphs": (_i32, [_vp, _i32]),
    "nnk_mob_solve": (_i32, [_vp, _vp, _vp, C.POINTER(SolveParams), _i32, C.POINTER(SolveInfo), _i32]),
    "nnk_mob_set_refinement": (_i32, [_vp, _vp, _i32, _f64]),
    "nnk_mob_apply_adjoint": (_i32, [_vp, _vp, _vp, _i32]),
    "nnk_mob_apply_fmm": (_i32, [_vp, _vp, _vp, _vp, _i32]),
    "nnk_mob_solve_adjoint": (_i32, [_vp, _vp, _vp, C.POINTER(SolveParams), C.POINTER(SolveInfo), _i32]),
    "nnk_mob_grad_positions": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32]),
    "nnk_mob_grad_eps": (_i32, [_vp, _vp, _vp, _vp, _pd, _i32]),
    "nnk_mob_destroy": (_i32, [_vp]),
    "nnk_batch_create": (_i32, [_vp, _i32, _vp, _vp, _vp, C.POINTER(FmmParams), _i32, C.POINTER(_vp)]),
    "nnk_batch_layout": (_i32, [_vp, _pi64, _vp]),
    "nnk_batch_apply": (_i32, [_vp, _vp, _vp, _i32]),
    "nnk_batch_solve": (_i32, [_vp, _vp, _vp, C.POINTER(SolveParams), _vp, _i32]),
    "nnk_batch_set_refinement": (_i32, [_vp, _i32, _i32, _f64]),
    "nnk_batch_matvecs": (_i32, [_vp, _pi64]),
    "nnk_batch_use_graphs": (_i32, [_vp, _i32]),
    "nnk_batch_set_deflation": (_i32, [_vp, _i32]),
    "nnk_batch_profile": (_i32, [_vp, _i32]),
    "nnk_batch_profile_read": (_i32, [_vp, _i32, _vp, _vp]),
    "nnk_batch_destroy": (_i32, [_vp]),
    "nnk_direct_nearest_noalloc": (_i32, [_i32, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _i64, _f64, _f64,
                                          _vp]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run: python stokes-nnkifmm_b200/build_lib.py")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class NNKError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class MaxDepthError(NNKError):
    pass


class NoConvergence(NNKError):
    pass


def check(rc, ctx=None, what=""):
    if rc == NNK_OK:
        return
    msg = lib.nnk_last_error(ctx).decode() if ctx else f"status {rc}"
    if rc == NNK_E_MAXDEPTH:
        raise MaxDepthError(rc, msg)
    if rc == NNK_E_NOCONV:
        raise NoConvergence(rc, msg)
    raise NNKError(rc, f"{what}: {msg}" if what else msg)


class Context:
    """One CUDA device and stream (nnk_ctx)."""

    _destroy = lib.nnk_ctx_destroy  # held by the class: module globals may be gone at exit

    def __init__(self, device=0):
        h = _vp()
        check(lib.nnk_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def set_stream(self, stream_ptr):
        check(lib.nnk_ctx_set_stream(self.h, _vp(stream_ptr)), self.h, "set_stream")

    def synchronize(self):
        check(lib.nnk_ctx_synchronize(self.h), self.h, "synchronize")

    def measure_l2_read(self):
        """L2 read bandwidth of this device in GB/s (nnk_measure_l2_read): a
        streaming read of an L2-resident buffer on this context's stream."""
        g = C.c_double()
        check(lib.nnk_measure_l2_read(self.h, C.byref(g)), self.h, "measure_l2_read")
        return g.value

    def __del__(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None


_contexts = {}


def context(device=0):
    if device not in _contexts:
        _contexts[device] = Context(device)
    return _contexts[device]


def ptr(a):
    """Raw pointer of a C-contiguous numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return a.data_ptr()
