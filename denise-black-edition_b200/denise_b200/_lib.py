"""ctypes binding of libdenise_b200.so (the C ABI in include/denise_b200.h).

The shared library is built in-tree by ``denise-black-edition_b200/build.py``.
Importing this module loads it; if it is missing the import fails loudly -
there is no CPU fallback for the propagator.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libdenise_b200.so")

DN_MAX_L = 5

DN_OK = 0
DN_EINVAL = -1
DN_ENOMEM = -2
DN_EUNSTABLE = -3
DN_ETIMEDOUT = -4
DN_EDEVICE = -5
DN_ENOTSUP = -6
DN_EIO = -7
DN_ESTATE = -8

ERROR_NAMES = {
    DN_EINVAL: "DN_EINVAL", DN_ENOMEM: "DN_ENOMEM", DN_EUNSTABLE: "DN_EUNSTABLE",
    DN_ETIMEDOUT: "DN_ETIMEDOUT", DN_EDEVICE: "DN_EDEVICE", DN_ENOTSUP: "DN_ENOTSUP",
    DN_EIO: "DN_EIO", DN_ESTATE: "DN_ESTATE",
}

MODE_FORWARD, MODE_ADJOINT, MODE_OBJECTIVE = 0, 1, 2
SNAP_F32, SNAP_F16, SNAP_BF16 = 0, 1, 2
ACC_F32, ACC_F64 = 0, 1
ARITH_EXACT, ARITH_FMA = 0, 1
KERN_PAIRED, KERN_COLUMN, KERN_VPIPE, KERN_FUSED = 0, 1, 2, 3
SEC_VX, SEC_VY, SEC_P, SEC_CURL, SEC_DIV = 0, 1, 2, 3, 4


class DeniseError(RuntimeError):
    """A DN_E* status returned by the library; ``code`` holds the value."""

    def __init__(self, code, msg):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("dh", ctypes.c_float), ("dt", ctypes.c_float),
        ("nt", ctypes.c_int), ("fdorder", ctypes.c_int), ("maxrelerror", ctypes.c_int),
        ("free_surf", ctypes.c_int), ("fw", ctypes.c_int),
        ("damping", ctypes.c_float), ("fpml", ctypes.c_float),
        ("npower", ctypes.c_float), ("k_max_pml", ctypes.c_float),
        ("boundary", ctypes.c_int), ("L", ctypes.c_int),
        ("fl", ctypes.c_float * DN_MAX_L), ("ts", ctypes.c_float),
        ("invmat1", ctypes.c_int), ("grad_form", ctypes.c_int), ("quelltypb", ctypes.c_int),
        ("seismo", ctypes.c_int), ("dtinv", ctypes.c_int), ("eprecond", ctypes.c_int),
        ("store_snapshots", ctypes.c_int), ("snap_precision", ctypes.c_int),
        ("grad_accum", ctypes.c_int), ("arith", ctypes.c_int), ("honor_q", ctypes.c_int),
        ("ckpt_steps", ctypes.c_int),
    ]


class Acq(ctypes.Structure):
    _fields_ = [
        ("nsrc", ctypes.c_int),
        ("src_i", ctypes.POINTER(ctypes.c_int)), ("src_j", ctypes.POINTER(ctypes.c_int)),
        ("src_type", ctypes.POINTER(ctypes.c_int)), ("src_azi", ctypes.POINTER(ctypes.c_float)),
        ("signals", ctypes.POINTER(ctypes.c_float)),
        ("ntr", ctypes.c_int),
        ("rec_i", ctypes.POINTER(ctypes.c_int)), ("rec_j", ctypes.POINTER(ctypes.c_int)),
    ]


class Pml(ctypes.Structure):
    _fields_ = [(n, ctypes.POINTER(ctypes.c_float)) for n in (
        "d_x", "K_x", "alpha_prime_x", "a_x", "b_x",
        "d_x_half", "K_x_half", "alpha_prime_x_half", "a_x_half", "b_x_half",
        "d_y", "K_y", "alpha_prime_y", "a_y", "b_y",
        "d_y_half", "K_y_half", "alpha_prime_y_half", "a_y_half", "b_y_half")]


PML_NAMES = [f[0] for f in Pml._fields_]


class Precond(ctypes.Structure):
    """dn_precond: smooth_grad and precond_PSV switches (the .inp keywords)."""
    _fields_ = [
        ("spatfilter", ctypes.c_int), ("wd_damp", ctypes.c_float), ("wd_damp1", ctypes.c_float),
        ("fc_end", ctypes.c_float), ("c_vs", ctypes.c_float),
        ("taper_vert", ctypes.c_int), ("taper_hor", ctypes.c_int), ("taper_sources", ctypes.c_int),
        ("taper_file", ctypes.c_int), ("gradt", ctypes.c_int * 4), ("exp_taper_grad_hor", ctypes.c_float),
        ("srtshape", ctypes.c_int), ("srtradius", ctypes.c_float), ("filtsize", ctypes.c_int),
        ("taper_vp", ctypes.POINTER(ctypes.c_float)), ("taper_vs", ctypes.POINTER(ctypes.c_float)),
        ("taper_rho", ctypes.POINTER(ctypes.c_float)),
        ("nsrc", ctypes.c_int), ("src_x", ctypes.POINTER(ctypes.c_float)), ("src_z", ctypes.POINTER(ctypes.c_float)),
        ("ntr", ctypes.c_int), ("rec_i", ctypes.POINTER(ctypes.c_int)), ("rec_j", ctypes.POINTER(ctypes.c_int)),
    ]


class ResidualOpts(ctypes.Structure):
    """dn_residual_opts: the calc_res options (LNORM, GRAD_FORM, MODE, N_ORDER, ...)."""
    _fields_ = [
        ("lnorm", ctypes.c_int), ("grad_form", ctypes.c_int), ("mode", ctypes.c_int), ("n_order", ctypes.c_int),
        ("comp_weight", ctypes.c_int), ("c_vp", ctypes.c_float), ("c_rho", ctypes.c_float),
        ("fc_start", ctypes.c_float), ("fc_end", ctypes.c_float), ("kill", ctypes.POINTER(ctypes.c_int)),
        ("offset_mute", ctypes.c_int), ("offsetc", ctypes.c_float), ("timewin", ctypes.c_int),
        ("gamma", ctypes.c_float), ("twlength_minus", ctypes.c_float), ("src_x", ctypes.c_float),
        ("src_z", ctypes.c_float),
    ]


class AccumOpts(ctypes.Structure):
    """dn_accum_opts: per-shot energy scaling and circular taper of the gradient assembly."""
    _fields_ = [
        ("energy", ctypes.c_int), ("c_vp", ctypes.c_float), ("c_vs", ctypes.c_float), ("c_rho", ctypes.c_float),
        ("circular_taper", ctypes.c_int), ("srtshape", ctypes.c_int), ("srtradius", ctypes.c_float),
        ("filtsize", ctypes.c_int), ("src_x", ctypes.c_float), ("src_z", ctypes.c_float),
    ]

# every function the header declares, with its argument types
_P = ctypes.POINTER
_c_int_p = _P(ctypes.c_int)
_c_float_p = _P(ctypes.c_float)
_c_double_p = _P(ctypes.c_double)
_vp = ctypes.c_void_p
SIGNATURES = {
    "dn_last_error": (ctypes.c_char_p, []),
    "dn_version": (ctypes.c_int, [_c_int_p, _c_int_p]),
    "dn_device_count": (ctypes.c_int, [_c_int_p]),
    "dn_holbergcoeff": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_float_p]),
    "dn_pml_profiles": (ctypes.c_int, [_P(Params), _P(Pml)]),
    "dn_cfl_check": (ctypes.c_int, [_P(Params), ctypes.c_float, _c_double_p]),
    "dn_average_materials": (ctypes.c_int, [_P(Params), _c_float_p, _c_float_p, _c_float_p,
                                            _c_float_p, _c_float_p, _c_float_p]),
    "dn_prepare_visc": (ctypes.c_int, [_P(Params)] + [_c_float_p] * 16),
    "dn_wavelet": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, ctypes.c_float, ctypes.c_int, _c_float_p]),
    "dn_wavelet_ex": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                     _c_float_p, ctypes.c_int, _c_float_p]),
    "dn_model_create": (ctypes.c_int, [_P(Params), _c_float_p, _c_float_p, _c_float_p,
                                       _c_float_p, _c_float_p, ctypes.c_int, _P(_vp)]),
    "dn_model_destroy": (ctypes.c_int, [_vp]),
    "dn_model_params": (ctypes.c_int, [_vp, _P(Params)]),
    "dn_model_footprint": (ctypes.c_int, [_P(Params), _P(ctypes.c_size_t)]),
    "dn_shot_footprint": (ctypes.c_int, [_P(Params), ctypes.c_int, ctypes.c_int, _P(ctypes.c_size_t)]),
    "dn_shot_create": (ctypes.c_int, [_vp, _P(Acq), _P(_vp)]),
    "dn_shot_destroy": (ctypes.c_int, [_vp]),
    "dn_run": (ctypes.c_int, [_P(_vp), ctypes.c_int, ctypes.c_int]),
    "dn_run_plain": (ctypes.c_int, [_vp, ctypes.c_int]),
    "dn_shot_get_sections": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p]),
    "dn_shot_set_residuals": (ctypes.c_int, [_vp, _c_float_p, _c_float_p, _c_float_p]),
    "dn_shot_accumulate_gradient": (ctypes.c_int, [_vp]),
    "dn_shot_accumulate_gradient_precond": (ctypes.c_int, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "dn_model_get_gradient": (ctypes.c_int, [_vp, _c_float_p, _c_float_p, _c_float_p]),
    "dn_model_zero_gradient": (ctypes.c_int, [_vp]),
    "dn_model_set_gradient": (ctypes.c_int, [_vp, _c_float_p, _c_float_p, _c_float_p]),
    "dn_precond_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_float, _P(Precond), ctypes.c_int,
                                         _P(_vp)]),
    "dn_precond_destroy": (ctypes.c_int, [_vp]),
    "dn_precond_apply": (ctypes.c_int, [_vp, _vp]),
    "dn_taper_coefficients": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_float, _P(Precond), ctypes.c_int,
                                             _c_float_p]),
    "dn_shot_accumulate_gradient_ex": (ctypes.c_int, [_vp, _P(AccumOpts)]),
    "dn_shot_get_field": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p]),
    "dn_run_steps": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "dn_shot_get_snapshot": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_float_p]),
    "dn_last_run_stats": (ctypes.c_int, [_c_double_p, _P(ctypes.c_longlong)]),
    "dn_profile_steps": (ctypes.c_int, [_P(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_double_p]),
    "dn_residual_l2": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                      _c_double_p]),
    "dn_shot_residual": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p, _c_double_p]),
    "dn_shot_rtm_source": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p]),
    "dn_tdfilt": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                 ctypes.c_float]),
    "dn_tdfilt_host": (ctypes.c_int, [_c_float_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_int]),
    "dn_shot_residual_ex": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p, _P(ResidualOpts), _c_double_p]),
    "dn_residual_ex": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                      _c_int_p, _c_int_p, _P(ResidualOpts), _c_double_p]),
    "dn_queue_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _P(_vp)]),
    "dn_queue_destroy": (ctypes.c_int, [_vp]),
    "dn_queue_add": (ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    "dn_queue_step": (ctypes.c_int, [_vp, _P(_vp), _c_int_p, ctypes.c_int, _c_int_p]),
    "dn_queue_count": (ctypes.c_int, [_vp, _c_int_p, _c_int_p]),
    "dn_set_tile_shape": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong,
                                         ctypes.c_int, ctypes.c_int]),
    "dn_clear_tile_shapes": (ctypes.c_int, []),
    "dn_get_tile_shape": (ctypes.c_int, [_P(Params), _c_int_p, _c_int_p]),
    "dn_set_kernel_rule": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                          ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "dn_get_kernel_choice": (ctypes.c_int, [_P(Params), _c_int_p, _c_int_p, _c_int_p]),
    "dn_shot_kernel": (ctypes.c_int, [_vp, _c_int_p, _c_int_p]),
    "dn_model_get_material": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p]),
    "dn_dot": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _c_double_p]),
    "dn_lbfgs_create": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, ctypes.c_int, _P(_vp)]),
    "dn_lbfgs_destroy": (ctypes.c_int, [_vp]),
    "dn_lbfgs_push": (ctypes.c_int, [_vp, _vp, _vp]),
    "dn_lbfgs_count": (ctypes.c_int, [_vp, _c_int_p]),
    "dn_lbfgs_direction": (ctypes.c_int, [_vp, _vp, _vp]),
    "dn_optim_create": (ctypes.c_int, [ctypes.c_int] * 6 + [_P(_vp)]),
    "dn_optim_destroy": (ctypes.c_int, [_vp]),
    "dn_optim_reset": (ctypes.c_int, [_vp]),
    "dn_optim_step": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _c_float_p]),
    "dn_optim_get": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p]),
    "dn_model_gradient_to_device": (ctypes.c_int, [_vp, _vp]),
    "dn_model_gradient_from_device": (ctypes.c_int, [_vp, _vp]),
    "dn_calc_opt_step": (ctypes.c_int, [_c_double_p, _c_float_p, _c_float_p]),
    "dn_mat_update": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [_c_float_p] * 6 + [ctypes.c_float, _c_float_p,
                                     ctypes.c_int, _c_int_p, ctypes.c_float] + [_c_float_p] * 4),
    "dn_device_memory": (ctypes.c_int, [ctypes.c_int, _P(ctypes.c_size_t), _P(ctypes.c_size_t)]),
    "dn_device_trim": (ctypes.c_int, [ctypes.c_int]),
    "dn_inp_read": (ctypes.c_int, [ctypes.c_char_p, _vp]),
    "dn_inp_nt": (ctypes.c_int, [_vp]),
    "dn_inp_params": (ctypes.c_int, [_vp, ctypes.c_float, _P(Params)]),
    "dn_read_model_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _c_float_p]),
    "dn_read_sources": (ctypes.c_int, [ctypes.c_char_p, _P(ctypes.c_int), _P(_c_float_p), _P(ctypes.c_float)]),
    "dn_read_signal_file": (ctypes.c_int, [ctypes.c_char_p, _P(ctypes.c_int), _P(_c_float_p)]),
    "dn_source_cell": (ctypes.c_int, [ctypes.c_float, ctypes.c_float, ctypes.c_float, _P(ctypes.c_int),
                                      _P(ctypes.c_int)]),
    "dn_read_receivers": (ctypes.c_int, [ctypes.c_char_p, _c_float_p, ctypes.c_float, _P(ctypes.c_int),
                                         _P(_P(ctypes.c_int)), _P(_P(ctypes.c_int))]),
    "dn_write_su": (ctypes.c_int, [ctypes.c_char_p, _c_float_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_float, ctypes.c_float, ctypes.c_float, _P(ctypes.c_int),
                                   _P(ctypes.c_int), _c_float_p, ctypes.c_float, ctypes.c_float]),
    "dn_write_seis": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _c_float_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P(ctypes.c_int),
                                     _P(ctypes.c_int), _c_float_p, ctypes.c_float, ctypes.c_float]),
    "dn_read_su": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _c_float_p]),
    "dn_forward_inp": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "dn_residual_l2_noalloc": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                              ctypes.c_int, _c_double_p]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python denise-black-edition_b200/build.py` "
            "(the propagator has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(code):
    if code != DN_OK:
        raise DeniseError(code, lib.dn_last_error().decode(errors="replace"))
    return code


def fptr(a):
    """float32 C-contiguous array -> float*; None -> NULL."""
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_c_float_p)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_c_int_p)


def device_count():
    n = ctypes.c_int(0)
    lib.dn_device_count(ctypes.byref(n))
    return n.value
