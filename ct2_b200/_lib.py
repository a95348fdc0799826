"""ctypes binding of libct2g.so (the C ABI declared in include/ct2g.h).

The library is the only compute path: if it is missing or cannot load, every
call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libct2g.so")

CT2G_OK = 0
SOFT_PLUMMER = 0
SOFT_SPHERE = 1
MAX_ORDER = 6


class Options(ctypes.Structure):
    _fields_ = [("bwidth", ctypes.c_float), ("hsoft", ctypes.c_float), ("eta", ctypes.c_float),
                ("GM", ctypes.c_float), ("mesh", ctypes.c_int), ("order", ctypes.c_int),
                ("kernel", ctypes.c_int), ("device", ctypes.c_int),
                ("max_particles", ctypes.c_size_t)]


class Tuning(ctypes.Structure):
    _fields_ = [("dense_cell", ctypes.c_int), ("near_blocks_per_sm", ctypes.c_int),
                ("fft_tile", ctypes.c_int), ("split_mg2l", ctypes.c_int),
                ("sparse_path", ctypes.c_int), ("overlap", ctypes.c_int),
                ("mg2l_greens_direct", ctypes.c_int), ("near_chunks_per_warp", ctypes.c_int),
                ("plane_pipe", ctypes.c_int), ("cols_tma", ctypes.c_int),
                ("x_tma", ctypes.c_int), ("p2m_compact", ctypes.c_int)]


STEP_GRAPH = 1
FFT_FP32, FFT_TC_BF16X3 = 0, 1
SELECT_NONE, SELECT_FIXED, SELECT_MLP, SELECT_ALL = 0, 1, 2, 3
MLP_NIN, MLP_NHID, MLP_NPARAM = 24, 64, 5825


class KickParams(ctypes.Structure):
    _fields_ = [("ascending", ctypes.c_int), ("descending", ctypes.c_int), ("top", ctypes.c_int),
                ("first", ctypes.c_int), ("rung", ctypes.c_int), ("t0", ctypes.c_float),
                ("eta", ctypes.c_float), ("max_dt", ctypes.c_float), ("scale", ctypes.c_float)]


# (name, restype, argtypes) for every symbol of include/ct2g.h
_P = ctypes.c_void_p
_I = ctypes.c_int
_SZ = ctypes.c_size_t
_F = ctypes.c_float
_D = ctypes.c_double
SYMBOLS = [
    ("ct2g_default_options", None, [_P]),
    ("ct2g_create", _I, [_P, _P]),
    ("ct2g_destroy", _I, [_P]),
    ("ct2g_last_error", ctypes.c_char_p, [_P]),
    ("ct2g_status_string", ctypes.c_char_p, [_I]),
    ("ct2g_get_options", _I, [_P, _P]),
    ("ct2g_set_params", _I, [_P, _F, _F, _F]),
    ("ct2g_upload_particles", _I, [_P, _P, _P, _P, _P, _P, _P, _P, _SZ]),
    ("ct2g_download_particles", _I, [_P, _P, _P, _P, _P, _P, _P, _P, _P]),
    ("ct2g_particle_count", _SZ, [_P]),
    ("ct2g_particle_to_grid", _I, [_P]),
    ("ct2g_download_cells", _I, [_P, _P, _P]),
    ("ct2g_compute_multipoles", _I, [_P]),
    ("ct2g_download_multipoles", _I, [_P, _P]),
    ("ct2g_compute_expansions", _I, [_P]),
    ("ct2g_download_expansions", _I, [_P, _P]),
    ("ct2g_download_greens", _I, [_P, _P]),
    ("ct2g_compute_forces", _I, [_P]),
    ("ct2g_download_forces", _I, [_P, _P, _P, _P, _P]),
    ("ct2g_upload_forces", _I, [_P, _P, _P, _P]),
    ("ct2g_kick_update", _I, [_P, _P, _P]),
    ("ct2g_kick", _I, [_P, _P, _P]),
    ("ct2g_drift", _I, [_P, _F, _F]),
    ("ct2g_kick_drift", _I, [_P, _P, _F, _F, _I, _P]),
    ("ct2g_kick_drift_host", _I, [_P, _P, _F, _F, _I] + [_P] * 7 + [_SZ] + [_P] * 9),
    ("ct2g_create_boxes", _I, [_P, _I, _P]),
    ("ct2g_set_boxes", _I, [_P, _P, _P]),
    ("ct2g_box_count", _I, [_P]),
    ("ct2g_batch_create", _I, [_P, _I, _P]),
    ("ct2g_batch_kick_drift", _I, [_P, _P, _F, _F, _P]),
    ("ct2g_batch_last_ms", _I, [_P, _P]),
    ("ct2g_batch_destroy", _I, [_P]),
    ("ct2g_get_tuning", _I, [_P, _P]),
    ("ct2g_set_tuning", _I, [_P, _P]),
    ("ct2g_autotune", _I, [_P, _P, _F, _F, ctypes.c_char_p, _P]),
    ("ct2g_learned_enable", _I, [_P, _F]),
    ("ct2g_learned_select", _I, [_P, _I, _F]),
    ("ct2g_learned_collect", _I, [_P, _P]),
    ("ct2g_learned_dataset", _I, [_P, _P, _P, _SZ, _P]),
    ("ct2g_learned_clear", _I, [_P]),
    ("ct2g_learned_cells", _I, [_P, _P, _P, _P, _P, _P, _SZ, _P, _P]),
    ("ct2g_mlp_init", _I, [_P, ctypes.c_uint64]),
    ("ct2g_mlp_set", _I, [_P, _P, _P, _P]),
    ("ct2g_mlp_get", _I, [_P, _P, _P, _P]),
    ("ct2g_mlp_train", _I, [_P, _I, _I, _F, ctypes.c_uint64, _I, _P]),
    ("ct2g_mlp_gradients", _I, [_P, _P, _P, _SZ, _P, _P]),
    ("ct2g_kick_step", _I, [_P, _P, _I, _D, _D, _D, _D, _I, _I, _P]),
    ("ct2g_sort_by_rung", _I, [_P, _I]),
    ("ct2g_push_rungs", _I, [_P]),
    ("ct2g_pop_rungs", _I, [_P]),
    ("ct2g_set_minrung", _I, [_P, _I]),
    ("ct2g_current_range", _I, [_P, _P, _P]),
    ("ct2g_rung_counts", _I, [_P, _P, _I, _P]),
    ("ct2g_fft_r2c_3d", _I, [_P, _P, _P, _I, _I]),
    ("ct2g_fft_c2r_3d", _I, [_P, _P, _P, _I, _I]),
    ("ct2g_fft3d_f32_dev", _I, [_P, _I, _P, _P, _I, _I]),
    ("ct2g_fft3d_c2c_f32_dev", _I, [_P, _I, _P, _I, _I]),
    ("ct2g_cic_deposit", _I, [_P, _I, _P]),
    ("ct2g_fft1d_real", _I, [_P, _P, _I, _I, _I]),
    ("ct2g_fft1d_complex", _I, [_P, _P, _I, _I, _I]),
    ("ct2g_scramble", _I, [_P, _P, _I, _I, _I]),
    ("ct2g_transpose_yz", _I, [_P, _P, _I]),
    ("ct2g_transpose_r2c", _I, [_P, _P, _P, _I]),
    ("ct2g_transpose_c2r", _I, [_P, _P, _P, _I]),
    ("ct2g_twiddles", _I, [_P, _I, _I, _P]),
    ("ct2g_ewald_direct", _I, [_P, _P, _P, _P, _SZ, _D, _D, _I, _P, _P]),
    ("ct2g_ewald_direct_noalloc", _I, [_I, _P, _P, _P, _SZ, _P, _P, _P, _SZ, _I, _D, _D, _D, _D,
                                       _I, _P, _P, _P]),
    ("ct2g_tc_selftest", _I, [_I, _P, _P, _I, _I, _P]),
    ("ct2g_wait_selftest", _I, [_P, ctypes.c_uint32]),
    ("ct2g_set_fft_mode", _I, [_P, _I]),
    ("ct2g_stream", _P, [_P]),
    ("ct2g_synchronize", _I, [_P]),
    ("ct2g_stage_times", _I, [_P, _P, _I]),
    ("ct2g_launch_count", ctypes.c_uint64, [_P]),
    ("ct2g_interaction_count", ctypes.c_uint64, [_P]),
]

_lib = None


def load():
    """Load libct2g.so, raising if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libct2g.so is not built (run python -m ct2_b200.build); "
                           "the gravity step has no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SYMBOLS:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class CT2GError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("ct2g status %d (%s): %s" % (status, _status_str(status), msg))
        self.status = status


def _status_str(s):
    try:
        return load().ct2g_status_string(s).decode()
    except Exception:  # pragma: no cover
        return "?"
