"""ctypes binding of libippi_lbm.so (include/ippi_lbm.h).

The library is built in-tree by ../build.py.  Loading fails loudly when it is
missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libippi_lbm.so")

IPPI_OK, IPPI_ERR_ARG, IPPI_ERR_CUDA, IPPI_ERR_DIVERGED, IPPI_ERR_STATE, IPPI_ERR_NOMEM = \
    0, -1, -2, -3, -4, -5
BGK, MRT, RR = 0, 1, 2
F64, F32, F16, BF16 = 0, 1, 2, 3
BC_REF_NEE, BC_CHANNEL = 0, 1
LES_NONE, LES_SMAGORINSKY, LES_LEARNED, LES_FIELD, LES_WALE, LES_CSM, LES_DYNAMIC = range(7)
MLP_PARAMS, MLP_STATS, MLP_GRAD_BLOCKS = 1313, 25, 296
ABI_VERSION = 3
DELTA_BILINEAR, DELTA_PESKIN4 = 0, 1
(FIELD_F, FIELD_RHO, FIELD_UX, FIELD_UY, FIELD_TAU, FIELD_AVG_U, FIELD_AVG_V, FIELD_AVG_RHO,
 FIELD_FLAGS, FIELD_NNFLAG) = range(10)

EXPORTS = ("ippi_abi_version", "ippi_params_default", "ippi_create", "ippi_destroy",
           "ippi_init_macros", "ippi_init_macros_f32", "ippi_download_f32", "ippi_set_les_cs", "ippi_set_learned_tensor_cores", "ippi_set_markers", "ippi_load_band_net", "ippi_step", "ippi_step_timed",
           "ippi_download", "ippi_forces", "ippi_force_history", "ippi_get_stream",
           "ippi_profile_steps", "ippi_last_error", "ippi_mass_noalloc", "ippi_load_tau_mlp",
           "ippi_filter_snapshot", "ippi_mlp_param_count", "ippi_mlp_scratch_floats", "ippi_mlp_grad",
           "ippi_mlp_adam", "ippi_mlp_forward", "ippi_set_tau_field", "ippi_load_tau_mlp_f32",
           "ippi_adjoint_forward", "ippi_adjoint_backward", "ippi_tau_scan", "ippi_tau_scan_state", "ippi_set_solid", "ippi_solid_force", "ippi_reequilibrate",
           "ippi_set_wall_distance", "ippi_diagnostics", "ippi_state_bytes", "ippi_save_state",
           "ippi_load_state")


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("collision", C.c_int), ("storage", C.c_int),
        ("bc_set", C.c_int), ("les_model", C.c_int), ("tau0", C.c_double), ("cs", C.c_double),
        ("u_in", C.c_double), ("rho0", C.c_double), ("plate_x0", C.c_int),
        ("avg_start", C.c_int), ("delta_kernel", C.c_int), ("mdf_iters", C.c_int),
        ("device", C.c_int),
    ]


class IppiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ippi error {code}: {msg}")
        self.code = code


class DivergedError(IppiError):
    pass


_lib = None
_dp = C.POINTER(C.c_double)


def lib() -> C.CDLL:
    """Load libippi_lbm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; run build.py (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        L.ippi_abi_version.restype = C.c_int
        if L.ippi_abi_version() != ABI_VERSION:
            raise ImportError(f"{LIB_PATH} has ABI {L.ippi_abi_version()}, expected {ABI_VERSION}; "
                              "rebuild it with build.py")
        L.ippi_params_default.argtypes = [C.POINTER(Params), C.c_int, C.c_int]
        L.ippi_params_default.restype = None
        L.ippi_create.argtypes = [C.POINTER(Params), C.POINTER(C.c_void_p)]
        L.ippi_destroy.argtypes = [C.c_void_p]
        L.ippi_init_macros.argtypes = [C.c_void_p, _dp, _dp, _dp]
        _fp = C.POINTER(C.c_float)
        L.ippi_init_macros_f32.argtypes = [C.c_void_p, _fp, _fp, _fp]
        L.ippi_download_f32.argtypes = [C.c_void_p, C.c_int, _fp, C.c_size_t]
        L.ippi_set_les_cs.argtypes = [C.c_void_p, C.c_double]
        L.ippi_set_learned_tensor_cores.argtypes = [C.c_void_p, C.c_int]
        L.ippi_set_markers.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.POINTER(C.c_int), _dp]
        L.ippi_load_band_net.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.c_size_t]
        L.ippi_step.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.ippi_step_timed.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.ippi_download.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        L.ippi_forces.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_int), _dp]
        L.ippi_force_history.argtypes = [C.c_void_p, _dp, C.c_int]
        L.ippi_get_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.ippi_profile_steps.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp]
        L.ippi_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        L.ippi_mass_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.ippi_load_tau_mlp.argtypes = [C.c_void_p, C.POINTER(C.c_uint16), C.c_size_t,
                                        C.POINTER(C.c_float), C.c_size_t]
        L.ippi_filter_snapshot.argtypes = [C.c_void_p, C.c_int, _dp, C.c_size_t]
        L.ippi_mlp_scratch_floats.restype = C.c_size_t
        _vp = C.c_void_p
        L.ippi_mlp_grad.argtypes = [_vp, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp]
        L.ippi_mlp_adam.argtypes = [_vp, _vp, _vp, _vp, C.c_int, C.c_float, C.c_float, C.c_float,
                                    C.c_float, _vp]
        L.ippi_mlp_forward.argtypes = [_vp, C.c_int, _vp, _vp, _vp]
        L.ippi_set_tau_field.argtypes = [C.c_void_p, _dp]
        L.ippi_load_tau_mlp_f32.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_size_t,
                                            C.POINTER(C.c_float), C.c_size_t]
        L.ippi_adjoint_forward.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.ippi_adjoint_backward.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.ippi_reequilibrate.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.ippi_set_wall_distance.argtypes = [C.c_void_p, _dp]
        L.ippi_diagnostics.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.ippi_state_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
        L.ippi_save_state.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.ippi_load_state.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_int)]
        L.ippi_set_solid.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), C.c_size_t]
        L.ippi_solid_force.argtypes = [C.c_void_p, _dp]
        L.ippi_tau_scan.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), _dp, C.c_int, C.c_int,
                                    C.c_double, _dp, _dp]
        L.ippi_tau_scan_state.argtypes = [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int,
                                          C.c_int, C.c_double, _vp, _vp, _vp]
        _lib = L
    return _lib


def last_error(h=None) -> str:
    buf = C.create_string_buffer(512)
    lib().ippi_last_error(h, buf, 512)
    return buf.value.decode(errors="replace")


def check(rc, h=None):
    if rc == IPPI_OK:
        return rc
    msg = last_error(h)
    if rc == IPPI_ERR_DIVERGED:
        raise DivergedError(rc, msg)
    raise IppiError(rc, msg)
