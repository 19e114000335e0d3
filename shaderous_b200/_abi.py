"""ctypes declarations of the C ABI in ``include/shaderous_b200.h``.

The library is loaded from the package directory (built in-tree by ``shaderous_b200.build``).
There is no fallback: if the shared library is missing or fails to load, importing the
simulation API raises.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libshaderous_b200.so"

SHZ_OK = 0
SHZ_E_CONFIG = -1
SHZ_E_OOM = -2
SHZ_E_NAN = -3
SHZ_E_CUDA = -4
SHZ_E_TIMEOUT = -5
SHZ_E_CANCELLED = -6
SHZ_E_NODEV = -7

BC_PERIODIC, BC_OUTFLOW, BC_REFLECT = 0, 1, 2
RECON = {"minmod": 0, "mc": 1, "vanleer": 2, "koren": 3, "ppm": 4}
RIEMANN = {"hllc": 0, "hll": 1}
PROBLEM = {"sod": 0, "kh": 1, "tgv": 2, "sedov": 3, "advect": 4, "blast": 5, "gauss": 6}
STOPPED = {0: "steps", 1: "time", 2: "end", 3: "timeout"}


class shz_config(C.Structure):
    _fields_ = [
        ("n", C.c_int32 * 3),
        ("dx", C.c_double),
        ("gamma", C.c_double),
        ("bc_lo", C.c_int32 * 3),
        ("bc_hi", C.c_int32 * 3),
        ("cfl", C.c_double),
        ("rho_floor", C.c_double),
        ("p_floor", C.c_double),
        ("eta_dual", C.c_double),
        ("shock_thresh", C.c_double),
        ("riemann", C.c_int32),
        ("recon", C.c_int32),
        ("isentropic", C.c_int32),
        ("signal_dims", C.c_int32),
        ("t_end", C.c_double),
        ("dt_max", C.c_double),
        ("device", C.c_int32),
    ]


class shz_run_opts(C.Structure):
    _fields_ = [("steps", C.c_int64), ("until", C.c_double), ("timeout_ms", C.c_double)]


class shz_run_result(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("dt", C.c_double),
        ("steps", C.c_int64),
        ("taken", C.c_int64),
        ("seconds", C.c_double),
        ("stopped", C.c_int32),
        ("last_dt", C.c_double),
    ]


class shz_diag(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("dt", C.c_double),
        ("steps", C.c_int64),
        ("mass", C.c_double),
        ("momentum", C.c_double * 3),
        ("e_kin", C.c_double),
        ("e_int", C.c_double),
        ("e_tot", C.c_double),
        ("max_mach", C.c_double),
        ("floored", C.c_double),
    ]


class shz_diag_ext(C.Structure):
    _fields_ = [("base", shz_diag), ("range", (C.c_double * 2) * 5), ("com", C.c_double * 3), ("e_grav", C.c_double),
                ("jeans_unresolved", C.c_double), ("nuclear_heating", C.c_double)]


class shz_problem(C.Structure):
    _fields_ = [("kind", C.c_int32), ("axis", C.c_int32), ("seed", C.c_uint64), ("a", C.c_double * 8)]


class shz_amr_config(C.Structure):
    _fields_ = [
        ("hydro", shz_config),
        ("ndim", C.c_int32),
        ("nr", C.c_int32),
        ("max_level", C.c_int32),
        ("cap", C.c_int32),
        ("box", C.c_double),
        ("refine_hi", C.c_double),
        ("refine_lo", C.c_double),
        ("regrid_every", C.c_int32),
        ("two_pass", C.c_int32),
        ("time_bins", C.c_int32),
        ("time_bins_always", C.c_int32),
    ]


class shz_mesh_spec(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("levels", C.c_void_p),
        ("coords", C.c_void_p),
        ("root_size", C.c_int32 * 3),
        ("block_size", C.c_int32 * 3),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("shift", C.c_int32),
    ]


class shz_request(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("n", C.c_int32),
        ("steps", C.c_int32),
        ("bc", C.c_int32),
        ("gamma", C.c_double),
        ("arrival", C.c_double),
        ("problem", shz_problem),
    ]


class shz_server_config(C.Structure):
    _fields_ = [
        ("hydro", shz_config),
        ("budget_bytes", C.c_double),
        ("max_grids", C.c_int32),
        ("round_steps", C.c_int32),
        ("keep_states", C.c_int32),
        ("direct_large", C.c_int32),
    ]


class shz_server_stats(C.Structure):
    _fields_ = [
        ("completed", C.c_int64),
        ("makespan_s", C.c_double),
        ("p50_s", C.c_double),
        ("p99_s", C.c_double),
        ("mean_s", C.c_double),
        ("zone_updates", C.c_double),
        ("zu_per_s", C.c_double),
        ("max_concurrent", C.c_int64),
        ("rounds", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("busy_s", C.c_double),
    ]


class shz_tune_entry(C.Structure):
    _fields_ = [(f, C.c_int32) for f in ("kernel", "ndim", "recon", "isentropic", "size_class", "variant", "per_sm", "tz",
                                         "candidates")] + [("ms", C.c_float), ("default_ms", C.c_float)]


class shz_profile_result(C.Structure):
    _fields_ = [("steps", C.c_int32), ("total_ms", C.c_double), ("sweep_ms", C.c_double), ("launches", C.c_int64)]


# (name, restype, argtypes): every entry point declared in include/shaderous_b200.h
SIGNATURES = [
    ("shz_config_default", C.c_int, [C.POINTER(shz_config), C.c_int32, C.c_int32, C.c_int32, C.c_double]),
    ("shz_create", C.c_int, [C.POINTER(shz_config), C.POINTER(C.c_void_p)]),
    ("shz_destroy", None, [C.c_void_p]),
    ("shz_last_error", C.c_char_p, [C.c_void_p]),
    ("shz_reset_problem", C.c_int, [C.c_void_p, C.POINTER(shz_problem)]),
    ("shz_problem_prims", C.c_int, [C.POINTER(shz_config), C.POINTER(shz_problem), C.c_int32, C.c_int32, C.c_void_p]),
    ("shz_set_state", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]),
    ("shz_get_state", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]),
    ("shz_step", C.c_int, [C.c_void_p, C.c_int32]),
    ("shz_run", C.c_int, [C.c_void_p, C.POINTER(shz_run_opts), C.POINTER(shz_run_result)]),
    ("shz_diagnostics", C.c_int, [C.c_void_p, C.POINTER(shz_diag)]),
    ("shz_diagnostics_ext", C.c_int, [C.c_void_p, C.POINTER(shz_diag_ext)]),
    ("shz_clock", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("shz_set_clock", C.c_int, [C.c_void_p, C.c_double, C.c_int64]),
    ("shz_set_t_end", C.c_int, [C.c_void_p, C.c_double]),
    ("shz_sync", C.c_int, [C.c_void_p]),
    ("shz_state_device", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    ("shz_profile", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(shz_profile_result)]),
    ("shz_reset_problem_slab", C.c_int, [C.c_void_p, C.POINTER(shz_config), C.POINTER(shz_problem), C.c_int32]),
    ("shz_halo_depth", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("shz_halo_device", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                  C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    ("shz_rate_device", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("shz_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("shz_kernel_launches", C.c_int64, [C.c_void_p]),
    ("shz_version", C.c_char_p, []),
    ("shz_tune_enable", C.c_int, [C.c_int32]),
    ("shz_tune_reset", None, []),
    ("shz_tune_entries", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("shz_selftest_wait_timeout", C.c_int, [C.c_int32, C.POINTER(C.c_int32)]),
    ("shz_tree_create", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_void_p)]),
    ("shz_tree_destroy", None, [C.c_void_p]),
    ("shz_tree_error", C.c_char_p, []),
    ("shz_tree_adapt", C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.POINTER(C.c_int32)]),
    ("shz_tree_last_steps", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("shz_tree_replay", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int32)]),
    ("shz_tree_refine", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("shz_tree_neighbor", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32)]),
    ("shz_tree_table", C.c_int, [C.c_void_p, C.c_void_p]),
    ("shz_tree_lists", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32)]),
    ("shz_tree_index_grid_size", C.c_int64, [C.c_void_p]),
    ("shz_tree_index_grid", C.c_int, [C.c_void_p, C.c_void_p]),
    ("shz_tree_index_grid_boxes", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("shz_tree_set_bc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("shz_tree_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("shz_amr_create", C.c_int, [C.POINTER(shz_amr_config), C.POINTER(C.c_void_p)]),
    ("shz_amr_destroy", None, [C.c_void_p]),
    ("shz_amr_error", C.c_char_p, [C.c_void_p]),
    ("shz_amr_reset_problem", C.c_int, [C.c_void_p, C.POINTER(shz_problem)]),
    ("shz_amr_step", C.c_int, [C.c_void_p, C.c_int32]),
    ("shz_amr_run", C.c_int, [C.c_void_p, C.POINTER(shz_run_opts), C.POINTER(shz_run_result)]),
    ("shz_amr_diagnostics", C.c_int, [C.c_void_p, C.POINTER(shz_diag)]),
    ("shz_amr_diagnostics_ext", C.c_int, [C.c_void_p, C.POINTER(shz_diag_ext)]),
    ("shz_amr_clock", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("shz_amr_regrid", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("shz_amr_leaves", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p]),
    ("shz_amr_table", C.c_int, [C.c_void_p, C.c_void_p]),
    ("shz_amr_get_leaves_state", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("shz_amr_flags", C.c_int, [C.c_void_p, C.c_void_p]),
    ("shz_amr_ghost_map", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    ("shz_amr_prims", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    ("shz_amr_regrid_table", C.c_int, [C.c_void_p, C.c_void_p]),
    ("shz_amr_profile", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(shz_profile_result)]),
    ("shz_amr_kernel_launches", C.c_int64, [C.c_void_p]),
    ("shz_amr_bins", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("shz_amr_bin_work", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int32)]),
    ("shz_amr_reset_mesh", C.c_int, [C.c_void_p, C.POINTER(shz_mesh_spec)]),
    ("shz_tune_pin", C.c_int, [C.c_int32, C.c_int32, C.c_int32]),
    ("shz_amr_set_leaves_state", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("shz_amr_set_clock", C.c_int, [C.c_void_p, C.c_double, C.c_int64]),
    ("shz_server_create", C.c_int, [C.POINTER(shz_server_config), C.POINTER(C.c_void_p)]),
    ("shz_server_destroy", None, [C.c_void_p]),
    ("shz_server_error", C.c_char_p, [C.c_void_p]),
    ("shz_server_submit", C.c_int, [C.c_void_p, C.POINTER(shz_request), C.POINTER(C.c_int64)]),
    ("shz_server_drain", C.c_int, [C.c_void_p, C.c_int32]),
    ("shz_server_run_stream", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(shz_server_stats)]),
    ("shz_server_cancel", C.c_int, [C.c_void_p, C.c_int64]),
    ("shz_server_poll", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    ("shz_server_result", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(shz_diag)]),
    ("shz_server_state", C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    ("shz_plain_run_stream", C.c_int, [C.POINTER(shz_server_config), C.c_void_p, C.c_int32, C.POINTER(shz_server_stats)]),
    ("shz_totals_noalloc", C.c_int, [C.POINTER(shz_config), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("shz_totals_noalloc_error", C.c_char_p, []),
]

SHZ_DIAG_VALUES = 9
SHZ_TOTALS_MAX_BLOCKS = 8192
SHZ_TOTALS_CELLS_PER_BLOCK = 16384

_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (raises OSError if it is not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OSError(f"{LIB_PATH} is not built: run `python -m shaderous_b200.build`")
        lib = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


NAN = math.nan
