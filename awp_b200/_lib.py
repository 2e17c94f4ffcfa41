"""Loader and ctypes signatures for libawpb200.so (include/awp_b200.h).

The library is built in-tree by ``make -C awp_b200/csrc`` (or
``__graft_entry__.build()``).  Importing this module never falls back to any
other implementation: a missing or unloadable library raises at once.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import CFUNCTYPE, POINTER, c_char_p, c_double, c_float, c_int, c_longlong, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libawpb200.so")

AWP_OK = 0
STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "CUDA error",
    3: "call out of order",
    4: "I/O error",
    5: "out of memory",
    6: "non-finite wavefield",
    7: "unsupported option",
}

# enum awp_field_id
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz",
          "r1", "r2", "r3", "r4", "r5", "r6",
          "d1", "mu", "lam", "qp", "qs",
          "sigma2", "cohes", "phi", "yldfac", "neta"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}


# int (*)(void* user, int set): the halo exchange hook of a sub-domain
EXCHANGE_FN = CFUNCTYPE(c_int, c_void_p, c_int)
HALO_VELOCITY, HALO_STRESS, HALO_MEDIA, HALO_YLDFAC, HALO_PLANES = 1, 2, 4, 8, 4

# int (*)(void* user, int first, int n, float* vx, float* vy, float* vz)
FRAME_READER = CFUNCTYPE(c_int, c_void_p, c_int, c_int, POINTER(c_float), POINTER(c_float),
                         POINTER(c_float))

class AwpError(RuntimeError):
    """A non-zero status returned by the library."""

    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: {STATUS.get(status, status)} ({detail})")
        self.status = status


class awp_params(ctypes.Structure):
    """Mirror of ``struct awp_params`` (pmcl3d command-line names)."""

    _fields_ = [
        ("nx", c_int), ("ny", c_int), ("nz", c_int),
        ("dh", c_float), ("dt", c_float),
        ("arbc", c_float), ("npc", c_int), ("nd", c_int),
        ("nve", c_int),
        ("fac", c_float), ("q0", c_float), ("ex", c_float), ("fp", c_float),
        ("socalq", c_int),
        ("ifault", c_int),
        ("nst", c_int),
        ("read_step", c_int),
        ("grid", c_int),
        ("ngrids", c_int),
    ]


_lib = None

_P = c_void_p
_F = POINTER(c_float)
_I = POINTER(c_int)
_D = POINTER(c_double)


def _sig(lib, name, res, args):
    fn = getattr(lib, name)
    fn.restype = res
    fn.argtypes = args
    return fn


def load() -> ctypes.CDLL:
    """Load the library once; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C awp_b200/csrc` "
            "(there is no fallback implementation)")
    lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
    pp = POINTER(awp_params)
    _sig(lib, "awp_params_default", None, [pp])
    _sig(lib, "awp_status_string", c_char_p, [c_int])
    _sig(lib, "awp_last_error", c_char_p, [])
    _sig(lib, "awp_ctx_create", c_int, [pp, POINTER(c_void_p)])
    _sig(lib, "awp_ctx_destroy", c_int, [_P])
    _sig(lib, "awp_set_stream", c_int, [_P, c_void_p])
    _sig(lib, "awp_padded_dims", c_int, [_P, POINTER(c_longlong)])
    _sig(lib, "awp_upload_media", c_int, [_P, c_int, _F])
    _sig(lib, "awp_upload_media_device", c_int, [_P, c_int, c_void_p])
    _sig(lib, "awp_upload_sources", c_int, [_P, c_int, _I, _F])
    _sig(lib, "awp_upload_plane_wave", c_int, [_P, c_int, c_void_p, c_void_p, c_void_p])
    _sig(lib, "awp_set_source_filter", c_int, [_P, c_int, _D, _D])
    _sig(lib, "awp_download_moment", c_int, [_P, _F])
    _sig(lib, "awp_upload_plasticity", c_int, [_P, _F, _F, _F, c_float, c_float, _F, _F])
    _sig(lib, "awp_step", c_int, [_P, c_int])
    _sig(lib, "awp_synchronize", c_int, [_P])
    _sig(lib, "awp_current_step", c_int, [_P, POINTER(c_longlong)])
    _sig(lib, "awp_field_download", c_int, [_P, c_int, _F])
    _sig(lib, "awp_field_upload", c_int, [_P, c_int, _F])
    _sig(lib, "awp_field_device_ptr", c_int, [_P, c_int, POINTER(c_void_p)])
    _sig(lib, "awp_gather_output", c_int,
         [_P] + [c_int] * 9 + [c_void_p] * 4)
    _sig(lib, "awp_compute_bathymetry", c_int, [_P, _I])
    _sig(lib, "awp_set_bathymetry", c_int, [_P, _I])
    _sig(lib, "awp_check_finite", c_int, [_P, _I])
    _sig(lib, "awp_mesh_create", c_int, [POINTER(awp_params), c_int, POINTER(c_void_p)])
    _sig(lib, "awp_mesh_destroy", c_int, [_P])
    _sig(lib, "awp_mesh_grid", c_int, [_P, c_int, POINTER(c_void_p)])
    _sig(lib, "awp_mesh_step", c_int, [_P, c_int])
    _sig(lib, "awp_mesh_synchronize", c_int, [_P])
    _sig(lib, "awp_set_subdomain", c_int, [_P, c_int, c_int])
    _sig(lib, "awp_halo_copy", c_int, [_P, c_int, c_int, c_int, c_int, c_void_p])
    _sig(lib, "awp_set_exchange", c_int, [_P, EXCHANGE_FN, c_void_p])
    _sig(lib, "awp_decomp_create", c_int, [POINTER(c_void_p), c_int, POINTER(c_void_p)])
    _sig(lib, "awp_decomp_step", c_int, [_P, c_int])
    _sig(lib, "awp_decomp_synchronize", c_int, [_P])
    _sig(lib, "awp_decomp_destroy", c_int, [_P])
    _sig(lib, "awp_decomp_set_stream", c_int, [_P, c_void_p])
    _sig(lib, "awp_mesh_set_stream", c_int, [_P, _P])
    _sig(lib, "awp_batch_create", c_int, [POINTER(c_void_p), c_int, POINTER(c_void_p)])
    _sig(lib, "awp_batch_destroy", c_int, [_P])
    _sig(lib, "awp_batch_step", c_int, [_P, c_int])
    _sig(lib, "awp_batch_synchronize", c_int, [_P])
    _sig(lib, "awp_batch_set_shape", c_int, [_P, c_int, c_int])
    _sig(lib, "awp_batch_get_shape", c_int, [_P, _I, _I])
    _sig(lib, "awp_batch_set_graph", c_int, [_P, c_int])
    _sig(lib, "awp_batch_set_mode", c_int, [_P, c_int])
    _sig(lib, "awp_batch_get_mode", c_int, [_P])
    _sig(lib, "awp_batch_set_branches", c_int, [_P, c_int])
    _sig(lib, "awp_batch_info", c_int, [_P, POINTER(c_longlong)])
    _sig(lib, "awp_receivers_init", c_int, [_P, c_char_p, c_longlong])
    _sig(lib, "awp_sgt_init", c_int, [_P, c_char_p, c_longlong])
    _sig(lib, "awp_receivers_count", c_int, [_P, _I])
    _sig(lib, "awp_sourcefile_init", c_int, [_P, c_char_p])
    _sig(lib, "awp_forcefile_init", c_int, [_P, c_char_p])
    _sig(lib, "awp_velocity_forcing_init", c_int,
         [_P, c_int, _I, c_int, c_int, c_int, FRAME_READER, c_void_p])
    _sig(lib, "awp_topo_metrics", c_int, [c_char_p, c_int, c_int, c_int, c_float, _F])
    _sig(lib, "awp_topography_init", c_int, [_P, c_char_p])
    _sig(lib, "awp_set_topo_plasticity", c_int, [_P, c_int])
    _sig(lib, "awp_set_moduli", c_int, [_P, _F, _F, _F])
    _sig(lib, "awp_reset", c_int, [_P])
    _sig(lib, "awp_seismograms", c_int, [_P, c_int, c_int, _I, _I, _F])
    _sig(lib, "awp_misfit_gradient", c_int,
         [_P, c_int, c_int, _I, _I, _F, c_int, POINTER(c_double), _F, _F, _F, _F])
    _sig(lib, "awp_misfit_gradient_q", c_int,
         [_P, c_int, c_int, _I, _I, _F, c_int, POINTER(c_double), _F, _F, _F, _F, _F, _F])
    _sig(lib, "awp_set_qinv", c_int, [_P, _F, _F])
    _sig(lib, "awp_adjoint_reserve", c_int, [_P, c_int, c_int])
    _sig(lib, "awp_adjoint_plan", c_int,
         [_P, c_int, c_int, _I, _I, _I, POINTER(c_double)])
    _sig(lib, "awp_input_read", c_int,
         [c_char_p, POINTER(c_longlong), c_char_p, c_int, _F, _F, _F, _I, c_longlong])
    _sig(lib, "awp_point_coefs", c_int,
         [c_char_p, c_int, c_int, c_int, c_int, c_float, c_longlong, _I, _I, _I, _I, _I,
          _F, _F, _F])
    _sig(lib, "awp_point_coefs_topo", c_int,
         [c_char_p, c_char_p, c_int, c_int, c_int, c_int, c_float, c_longlong, _I, _I, _I, _I,
          _I, _F, _F, _F])
    _sig(lib, "awp_device_bytes", c_int, [_P, POINTER(c_longlong)])
    _sig(lib, "awp_profile_phases", c_int, [_P, c_int])
    _sig(lib, "awp_phase_times", c_int, [_P, POINTER(c_double), POINTER(c_longlong)])
    _sig(lib, "awp_kernel_launches", c_int, [_P, POINTER(c_longlong)])
    _sig(lib, "awp_set_tuning", c_int, [c_char_p, c_int])
    _sig(lib, "awp_get_tuning", c_int, [c_char_p])
    _sig(lib, "awp_q_tau", c_int, [c_float, c_float, _F, _F, _F])
    _sig(lib, "awp_q_weights", c_int, [c_float, c_float, _F, _F])
    _sig(lib, "awp_cerjan", c_int,
         [c_float, c_int, c_int, c_int, c_int, c_int, c_int, _F, _F, _F])
    _sig(lib, "awp_texture_at", c_int,
         [_F, _F, c_float, c_int, c_int, c_int, c_int, c_int, c_int, c_int,
          _F, _F, _I, _F])
    # reference-named launchers (kernel_launch.h)
    _sig(lib, "SetDeviceConstValue", None,
         [_F, c_float, _I, _I, _I, c_int, c_float, c_float, _F, _F])
    _sig(lib, "SetDeviceFilterParameters", None, [c_int, _D, _D])
    _sig(lib, "dvelcx_H_opt", None, [c_void_p] * 13 + [c_int, c_int, c_void_p] + [c_int] * 4)
    _sig(lib, "dstrqc_H", None,
         [c_void_p] * 23 + [c_int, c_int, c_void_p] + [c_void_p] * 5 + [c_int] * 9)
    _sig(lib, "dstrqc_H_new", None,
         [c_void_p] * 23 + [c_int, c_int, c_void_p] + [c_void_p] * 5 + [c_int] * 9)
    _sig(lib, "fstr_H", None, [c_void_p] * 3 + [c_void_p] + [c_int] * 4)
    _sig(lib, "drprecpc_calc_H_opt", None, [c_void_p] * 13 + [c_int] * 5 + [c_void_p, c_int])
    _sig(lib, "drprecpc_app_H", None, [c_void_p] * 9 + [c_int] * 5 + [c_void_p, c_int])
    _sig(lib, "addsrc_H", None, [c_int, c_int, c_int, c_void_p, c_int, c_void_p] + [c_void_p] * 12 + [c_int])
    _sig(lib, "addkinsrc_H", None, [c_int, c_int, c_void_p, c_int, c_void_p] + [c_void_p] * 15 + [c_int])
    _sig(lib, "velbuffer_H", None,
         [c_void_p] * 8 + [c_int] * 13 + [c_void_p, c_int, c_void_p, c_int])
    _sig(lib, "awp_compat_exit_on_error", None, [c_int])
    _sig(lib, "awp_compat_last_error", c_int, [])
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != AWP_OK:
        detail = load().awp_last_error().decode(errors="replace")
        raise AwpError(status, where, detail)


# exported symbol names that include/awp_b200.h declares
def declared_symbols(header: str | None = None) -> list[str]:
    import re
    header = header or os.path.join(HERE, "..", "include", "awp_b200.h")
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"\btypedef\b[^;]*;", "", text)  # callback types declare no symbol
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)
    skip = {"if", "for", "while", "return", "sizeof", "defined"}
    out = []
    for n in names:
        if n in skip or n.startswith("AWP_B200_H"):
            continue
        if n not in out:
            out.append(n)
    return out
