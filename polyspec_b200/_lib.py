"""ctypes binding of libpscuda.so (the C ABI declared in include/pscuda.h).

The library is built in-tree by ``python -m polyspec_b200.build`` (or
``__graft_entry__.build()``).  There is no CPU fallback: if the library is
missing or cannot be loaded, importing the CUDA backend raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpscuda.so")

PS_OK = 0
PS_ERR_UNSUPPORTED = -2
PS_ERR_NOMEM = -3
PS_ERR_NOT_CONVERGED = -6
PS_PREC_FP64 = 0
PS_PREC_MIXED = 1

_c_int, _c_int64, _c_double, _c_size_t, _c_void_p = (ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                                                      ctypes.c_size_t, ctypes.c_void_p)

# name -> (restype, argtypes); every entry point declared in include/pscuda.h
SIGNATURES = {
    "ps_error_string": (ctypes.c_char_p, [_c_int]),
    "ps_version": (_c_int, []),
    "ps_device_sm_count": (_c_int, [ctypes.POINTER(_c_int)]),
    "ps_plan_create": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, ctypes.POINTER(_c_void_p)]),
    "ps_plan_destroy": (_c_int, [_c_void_p]),
    "ps_plan_info": (_c_int, [_c_void_p, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int),
                              ctypes.POINTER(_c_int64), ctypes.POINTER(_c_int64)]),
    "ps_plan_error_flag": (_c_int, [_c_void_p, ctypes.POINTER(_c_int), _c_int]),
    "ps_sht_workspace_bytes": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_synthesis": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_void_p, _c_size_t,
                              _c_void_p]),
    "ps_adjoint": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_double, _c_void_p,
                            _c_size_t, _c_void_p]),
    "ps_synthesis_noalloc": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_void_p]),
    "ps_plan_band": (_c_int, [_c_void_p, _c_int, ctypes.POINTER(_c_void_p)]),
    "ps_plan_set_tile": (_c_int, [_c_void_p, _c_int, _c_int, _c_int]),
    "ps_plan_set_table_format": (_c_int, [_c_void_p, _c_int]),
    "ps_plan_table_bytes": (_c_int, [_c_void_p, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_plan_build_table": (_c_int, [_c_void_p, _c_int, _c_void_p]),
    "ps_plan_has_table": (_c_int, [_c_void_p, _c_int, ctypes.POINTER(_c_int)]),
    "ps_plan_drop_tables": (_c_int, [_c_void_p]),
    "ps_roundtrip_workspace_bytes": (_c_int, [_c_void_p, _c_int, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_sht_weighted_roundtrip": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int64, _c_int, _c_int, _c_void_p,
                                           _c_void_p, _c_double, _c_void_p, _c_size_t, _c_void_p]),
    "ps_legendre_workspace_bytes": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_legendre_synthesis": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_void_p, _c_size_t,
                                       _c_void_p]),
    "ps_legendre_adjoint": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_double, _c_void_p,
                                     _c_size_t, _c_void_p]),
    "ps_pix_product": (_c_int, [_c_int, ctypes.POINTER(_c_void_p), _c_int, _c_void_p, _c_int64, _c_int, _c_double,
                                _c_void_p]),
    "ps_pix_radial_sum_workspace_bytes": (_c_int, [_c_int, _c_int64, ctypes.POINTER(_c_size_t)]),
    "ps_pix_radial_sum": (_c_int, [_c_int, _c_void_p, _c_void_p, ctypes.POINTER(_c_void_p), _c_int, _c_int, _c_int64,
                                   _c_void_p, _c_void_p, _c_size_t, _c_void_p]),
    "ps_apply_fl_weights": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, _c_void_p, _c_void_p, _c_int64, _c_double,
                                     _c_void_p, _c_void_p]),
    "ps_radial_sum_lm": (_c_int, [_c_void_p, _c_int, _c_void_p, _c_void_p, _c_int, _c_int, _c_int, _c_void_p,
                                  _c_int64, _c_void_p, _c_void_p]),
    "ps_outer_product_workspace_bytes": (_c_int, [_c_int, _c_int, _c_int64, ctypes.POINTER(_c_size_t)]),
    "ps_outer_product": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int, _c_int64, _c_int, _c_void_p, _c_void_p,
                                  _c_size_t, _c_void_p]),
    "ps_lbp_dims": (_c_int, [ctypes.POINTER(_c_int)] * 4),
    "ps_lbp_moments": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int,
                                _c_int64, _c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "ps_lbp_loss_grad": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, ctypes.c_float, _c_void_p,
                                  _c_void_p, _c_void_p, _c_void_p]),
    "ps_lbp_apply": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int,
                              _c_int64, _c_void_p]),
    "ps_mlp_dense_forward": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_int, _c_int, _c_void_p,
                                      _c_void_p]),
    "ps_mlp_dense_backward_workspace_bytes": (_c_int, [_c_int, _c_int, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_mlp_dense_backward": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_int, _c_int,
                                       _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_size_t, _c_void_p]),
    "ps_mlp_adam": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, ctypes.c_float,
                             ctypes.c_float, ctypes.c_float, ctypes.c_float, _c_int, _c_void_p]),
    "ps_lm_matvec3": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int64, _c_void_p]),
    "ps_lm_dot_workspace_bytes": (_c_int, [_c_int, _c_int64, ctypes.POINTER(_c_size_t)]),
    "ps_kint_bessel_table": (_c_int, [_c_void_p, _c_int64, _c_int, _c_int, _c_void_p, _c_void_p]),
    "ps_kint_radial": (_c_int, [_c_void_p, _c_void_p, _c_int64, _c_int, _c_int, _c_void_p, _c_int, _c_void_p,
                                _c_int, _c_void_p, _c_int, _c_int, _c_void_p, _c_int, _c_int, _c_int, _c_int, _c_int,
                                _c_int, _c_int, _c_void_p, _c_void_p]),
    "ps_gl_nodes": (_c_int, [_c_int, _c_void_p, _c_void_p, _c_void_p]),
    "ps_wigner_binned": (_c_int, [_c_void_p, _c_int, _c_int, _c_void_p, _c_int, _c_void_p, _c_int, _c_void_p,
                                  _c_void_p]),
    "ps_bispec_ideal_contract": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int, _c_int, _c_void_p, _c_int,
                                          _c_void_p, _c_void_p]),
    "ps_gaunt_table": (_c_int, [_c_void_p, _c_int, _c_int, _c_void_p, _c_void_p]),
    "ps_pF_map_real": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int, _c_void_p, _c_int, _c_int, _c_int, _c_int,
                                _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int64, _c_int, _c_int, _c_int,
                                _c_void_p, _c_void_p]),
    "ps_product_pnmu_sym": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int64, _c_void_p, _c_void_p, _c_void_p, _c_int,
                                     _c_void_p, _c_void_p]),
    "ps_product_q_complex": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int, _c_int64, _c_void_p, _c_void_p,
                                      _c_void_p, _c_int, _c_void_p, _c_void_p]),
    "ps_kint_collider_jlK": (_c_int, [_c_void_p, _c_void_p, _c_int64, _c_int, _c_void_p, _c_int, _c_void_p, _c_int,
                                      _c_void_p, _c_void_p]),
    "ps_kint_collider_F": (_c_int, [_c_void_p, _c_int, _c_int, _c_void_p, _c_int, _c_void_p, _c_int, _c_int, _c_int,
                                    _c_int, _c_int, _c_void_p, _c_void_p]),
    "ps_tau_collider_workspace_bytes": (_c_int, [_c_int64, ctypes.POINTER(_c_size_t)]),
    "ps_tau_sum_collider_diag": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_void_p, _c_void_p, _c_int, _c_int, _c_int,
                                          _c_void_p, _c_int, _c_void_p, _c_int, _c_double, _c_double, _c_void_p,
                                          _c_void_p, _c_size_t, _c_void_p]),
    "ps_tau_sum_collider_general": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                             _c_int, _c_int, _c_int, _c_int, _c_int, _c_void_p, _c_int, _c_int,
                                             _c_void_p, _c_int, _c_int, _c_int, _c_void_p, _c_void_p, _c_void_p,
                                             _c_size_t, _c_void_p]),
    "ps_convolve_F_collider": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int,
                                        _c_int, _c_int, _c_int, _c_void_p, _c_int, _c_int, _c_int, _c_void_p,
                                        _c_void_p, _c_int, _c_int, _c_int, _c_void_p, _c_void_p, _c_void_p,
                                        _c_void_p]),
    "ps_pF_map_complex": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int, _c_void_p, _c_int, _c_int, _c_int, _c_int,
                                   _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int64, _c_int, _c_int, _c_int,
                                   _c_void_p, _c_void_p]),
    "ps_tau_general_workspace_bytes": (_c_int, [_c_int, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_gaunt_row_table": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int, _c_int, _c_int, _c_void_p, _c_void_p]),
    "ps_tau_sum_general": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_int,
                                    _c_int, _c_void_p, _c_int, _c_int, _c_void_p, _c_int, _c_int, _c_int, _c_int,
                                    _c_void_p, _c_void_p, _c_void_p, _c_size_t, _c_void_p]),
    "ps_convolve_F_general": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int,
                                       _c_int, _c_int, _c_void_p, _c_int, _c_int, _c_int, _c_void_p, _c_void_p,
                                       _c_int, _c_int, _c_int, _c_int, _c_int, _c_void_p, _c_void_p, _c_void_p,
                                       _c_void_p]),
    "ps_shift_weight_workspace_bytes": (_c_int, [_c_int64, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_shift_weight_map_all": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, _c_int, _c_void_p, _c_int64, _c_void_p,
                                         _c_void_p, _c_int, _c_void_p, _c_void_p, _c_int64, _c_int, _c_int,
                                         _c_double, _c_double, _c_int, _c_void_p, _c_void_p, _c_void_p, _c_size_t,
                                         _c_void_p]),
    "ps_quad_triple": (_c_int, [_c_void_p, _c_int, _c_void_p, _c_int, _c_void_p, _c_int, _c_void_p, _c_int,
                                _c_void_p, _c_int, _c_void_p, _c_void_p]),
    "ps_healpix_neighbours": (_c_int, [_c_int, _c_void_p, _c_void_p, _c_void_p]),
    "ps_inpaint_average": (_c_int, [_c_void_p, _c_void_p, _c_int64, _c_void_p, _c_int64, _c_int, _c_void_p,
                                    _c_void_p]),
    "ps_tau_F_integral": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, _c_int, _c_int, _c_double, _c_double,
                                   _c_void_p, _c_void_p, _c_void_p]),
    "ps_tau_convolve_workspace_bytes": (_c_int, [_c_int64, ctypes.POINTER(_c_size_t)]),
    "ps_tau_convolve_F": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_void_p,
                                   _c_int, _c_int64, _c_void_p, _c_void_p, _c_void_p, _c_size_t, _c_void_p]),
    "ps_bispec_triplet_sums_workspace_bytes": (_c_int, [_c_int, _c_int64, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_bispec_triplet_sums": (_c_int, [_c_void_p, _c_int, _c_int64, _c_void_p, _c_void_p, _c_int, _c_void_p,
                                        _c_void_p, _c_size_t, _c_void_p]),
    "ps_bispec_pair_products": (_c_int, [_c_void_p, _c_int, _c_void_p, _c_int, _c_int64, _c_void_p, _c_void_p,
                                         _c_int, _c_void_p, _c_void_p]),
    "ps_bispec_assemble_q": (_c_int, [_c_void_p, _c_void_p, _c_int, _c_int64, _c_void_p, _c_void_p, _c_int,
                                      _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_void_p, _c_void_p,
                                      _c_void_p]),
    "ps_lm_dot": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int64, _c_void_p, _c_void_p, _c_size_t,
                           _c_void_p]),
    "ps_batch_workspace_bytes": (_c_int, [_c_void_p, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_batch_submit": (_c_int, [_c_void_p, _c_int, _c_void_p, _c_size_t, _c_void_p]),
    "ps_lm_matvec3_add": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int64, _c_void_p]),
    "ps_lm_quad_dot": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int64, _c_void_p, _c_void_p, _c_size_t,
                                _c_void_p]),
    "ps_cg_xr_update": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int64,
                                 _c_void_p]),
    "ps_cg_direction": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int64, _c_void_p]),
    "ps_cutprec_create": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_void_p, _c_void_p, _c_void_p,
                                   _c_void_p, ctypes.POINTER(_c_void_p)]),
    "ps_cutprec_destroy": (_c_int, [_c_void_p]),
    "ps_cutprec_workspace_bytes": (_c_int, [_c_void_p, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_cutprec_apply": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_int, _c_void_p, _c_size_t, _c_void_p]),
    "ps_cg_create": (_c_int, [_c_void_p, _c_int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_double,
                              ctypes.POINTER(_c_void_p)]),
    "ps_cg_destroy": (_c_int, [_c_void_p]),
    "ps_cg_workspace_bytes": (_c_int, [_c_void_p, _c_int, ctypes.POINTER(_c_size_t)]),
    "ps_cg_solve": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_int, _c_double,
                             ctypes.POINTER(_c_int), ctypes.POINTER(_c_double), _c_void_p, _c_size_t, _c_void_p]),
    "ps_stats_enable_timing": (_c_int, [_c_int]),
    "ps_stats_reset": (_c_int, []),
    "ps_stats_get": (_c_int, [_c_int, ctypes.POINTER(_c_int64), ctypes.POINTER(_c_double),
                              ctypes.POINTER(_c_double), ctypes.POINTER(_c_double)]),
}



class WorkItem(ctypes.Structure):
    """ps_work_item of ps_batch_submit (one single-map transform)."""
    _fields_ = [("plan", _c_void_p), ("direction", _c_int), ("spin", _c_int), ("inp", _c_void_p),
                ("out", _c_void_p), ("scale", _c_double)]


PS_DIR_SYNTHESIS = 0
PS_DIR_ADJOINT = 1

# pixel-product ops and radial-sum kinds (enums of include/pscuda.h, in order)
PIX_OPS = ["multiply", "multiply_asym", "multiplyC", "multiplyC_asym", "multiplyCC", "multiplyCC_asym", "multiply2",
           "multiply2R", "multiply2C", "multiplyRC", "multiplyRCstar", "multiplyRC_sym", "multiplyRCstar_sym",
           "multiplyRR", "multiplyRR_sym", "r2c", "r2cstar", "lens_phi_sum", "lens_phi_sum_sym",
           "product_real1", "product_real2"]
SUM_KINDS = ["gnl_loc_sum", "gnl_loc_disc_sum", "gnl_con_sum", "gnl_con_disc_sum", "gnl_dotdot_sum",
             "gnl_dotdot_disc_sum", "gnl_dotdel_sum", "gnl_dotdel_disc_sum", "gnl_deldel_sum", "gnl_deldel_disc_sum"]

KERNEL_KINDS = {"leg_synth": 0, "leg_adjoint": 1, "fft_synth": 2, "fft_adjoint": 3, "layout": 4, "pixel": 5,
                "vector": 6, "mlp": 7}


def stats(kind):
    """(launches, device ms when timing is on, algorithmic flops, algorithmic bytes) of one kernel kind."""
    n = _c_int64()
    ms = _c_double()
    fl = _c_double()
    by = _c_double()
    call("ps_stats_get", KERNEL_KINDS[kind] if isinstance(kind, str) else int(kind), ctypes.byref(n),
         ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(by))
    return int(n.value), float(ms.value), float(fl.value), float(by.value)

_lib = None


class PSError(RuntimeError):
    def __init__(self, func, code):
        msg = lib().ps_error_string(code).decode() if _lib is not None else str(code)
        super().__init__("%s failed: %s (%d)" % (func, msg, code))
        self.code = code


def lib():
    """Load libpscuda.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libpscuda.so is not built: run `python -m polyspec_b200.build` "
                          "(the CUDA backend has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(func, code):
    if code != PS_OK:
        raise PSError(func, code)
    return code


def call(name, *args):
    return check(name, getattr(lib(), name)(*args))
