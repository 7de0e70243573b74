"""ctypes binding of libchapsim.so (the sm_100a CUDA library) and of its C ABI.

The shared library is built in-tree (chapsim1ww_b200/libchapsim.so) by
``chapsim1ww_b200.build.build()``.  There is no CPU fallback: importing a
symbol from a missing library raises immediately.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchapsim.so")

CHAPSIM_OK = 0
ERRORS = {
    1: "CHAPSIM_ERR_ARG", 2: "CHAPSIM_ERR_CUDA", 3: "CHAPSIM_ERR_NOMEM", 4: "CHAPSIM_ERR_STATE",
    5: "CHAPSIM_ERR_NUMERIC", 6: "CHAPSIM_ERR_UNSUPPORTED", 7: "CHAPSIM_ERR_NODEVICE",
}
ITG, IIO = 1, 2
FP64, MIXED = 0, 1
F_U, F_V, F_W, F_P, F_PHI, F_RHSPHI, F_H0U, F_H0V, F_H0W = range(9)
R_DIVMAX, R_BULK, R_NANCOUNT = 0, 1, 2
PHASES = ["rhs", "adix", "adiz", "adiy", "fftx", "fftz", "ysolve", "ifftz", "ifftx", "corr"]


class ChapsimConfig(ctypes.Structure):
    """Mirror of ``chapsim_config`` in include/chapsim.h."""
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("lx", ctypes.c_double), ("lz", ctypes.c_double), ("str2", ctypes.c_double),
        ("istr2", ctypes.c_int32), ("flowdrvtp", ctypes.c_int32),
        ("ren", ctypes.c_double), ("dt", ctypes.c_double), ("cfgv", ctypes.c_double),
        ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
    ]


class ChapsimIOConfig(ctypes.Structure):
    """Mirror of ``chapsim_io_config`` in include/chapsim.h."""
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("thermal", ctypes.c_int32), ("prt", ctypes.c_double),
        ("qw_bot", ctypes.c_double), ("qw_top", ctypes.c_double), ("gravdir", ctypes.c_int32),
        ("visc_scheme", ctypes.c_int32), ("f_a", ctypes.c_double),
        ("coupled", ctypes.c_int32), ("isothermal", ctypes.c_int32),
        ("bcx_in", ctypes.c_int32), ("bcx_out", ctypes.c_int32),
    ]


# IO domain field and reduction ids
F_GX, F_GY, F_GZ, F_G0X, F_G0Y, F_G0Z = 10, 11, 12, 13, 14, 15
F_H, F_T, F_RHO, F_MU, F_K, F_RHOH, F_RHO0, F_MU0, F_DRHO, F_RHSE0 = range(16, 26)
R_DIVMAX_Q, R_BULK_G, R_BULK_H, R_BADCELLS, R_CFL = 3, 4, 5, 6, 7

# (name, restype, argtypes) for every symbol declared in include/chapsim.h
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
# coupled inflow/outflow ghost planes of an IO context (CHAPSIM_P_*), each (nz, ny + 2)
IO_PLANES = {n: q for q, n in enumerate((
    "in_u", "in_v", "in_w", "in_gx", "in_gy", "in_gz", "in_p", "in_rho",
    "out_u", "out_v", "out_w", "out_gx", "out_gy", "out_gz", "out_rho", "out_rhoh", "out_h", "out_t", "out_mu",
    "out_k", "conv0_x", "conv0_y", "conv0_z", "conv0_eng"))}
IO_BC_SCALARS = ("u_outlet", "scaling", "balance", "inflow", "outflow", "mass_rate", "u_outlet_eng")

SIGNATURES = [
    ("chapsim_config_default", _I, [ctypes.POINTER(ChapsimConfig)]),
    ("chapsim_create", _I, [ctypes.POINTER(ChapsimConfig), ctypes.POINTER(_P)]),
    ("chapsim_destroy", _I, [_P]),
    ("chapsim_last_error", ctypes.c_char_p, [_P]),
    ("chapsim_sync", _I, [_P]),
    ("chapsim_field_len", _I64, [_P]),
    ("chapsim_set_field", _I, [_P, _I, _I, _P, _I64]),
    ("chapsim_get_field", _I, [_P, _I, _I, _P, _I64]),
    ("chapsim_set_field_async", _I, [_P, _I, _I, _P, _I64]),
    ("chapsim_get_field_async", _I, [_P, _I, _I, _P, _I64]),
    ("chapsim_io_bc_inlet", _I, [_P, _P]),
    ("chapsim_io_bc_outlet_mom", _I, [_P, _I]),
    ("chapsim_io_bc_outlet_eng", _I, [_P, _I]),
    ("chapsim_io_set_plane", _I, [_P, _I, _P, _I64]),
    ("chapsim_io_get_plane", _I, [_P, _I, _P, _I64]),
    ("chapsim_io_bc_scalars", _I, [_P, _P, _I]),
    ("chapsim_set_field_device", _I, [_P, _I, _I, _P, _I64]),
    ("chapsim_get_field_device", _I, [_P, _I, _I, _P, _I64]),
    ("chapsim_get_mesh", _I, [_P, _I, _P, _I64]),
    ("chapsim_init_random", _I, [_P, ctypes.c_uint64, _D, _I]),
    ("chapsim_rk3_mom_tg", _I, [_P, _I]),
    ("chapsim_step_tg", _I, [_P, _I]),
    ("chapsim_divg", _I, [_P, _I, _I]),
    ("chapsim_pois3d", _I, [_P, _I]),
    ("chapsim_velo_correction", _I, [_P, _I, _I]),
    ("chapsim_reduce", _I, [_P, _I, _I, _DP]),
    ("chapsim_get_stream", _I, [_P, ctypes.POINTER(_P)]),
    ("chapsim_phase_timing", _I, [_P, _I]),
    ("chapsim_phase_times", _I, [_P, _DP, _I, ctypes.POINTER(_I64)]),
    ("chapsim_phase_reset", _I, [_P]),
    ("chapsim_launch_count", _I, [_P, ctypes.POINTER(_I64)]),
    ("chapsim_launch_count_reset", _I, [_P]),
    ("chapsim_set_tuning", _I, [_P, _I, _I]),
    ("chapsim_get_tuning", _I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    ("chapsim_set_line_tuning", _I, [_P, _I]),
    ("chapsim_io_wall_values", _I, [_P, _DP, _I]),
    ("chapsim_get_line_tuning", _I, [_P, ctypes.POINTER(_I)]),
    ("chapsim_props_create", _I, [_P, _P, _P, _P, _P, _P, _I, _I, ctypes.POINTER(_P)]),
    ("chapsim_props_destroy", _I, [_P]),
    ("chapsim_props_last_error", ctypes.c_char_p, [_P]),
    ("chapsim_props_update", _I, [_P, _I, _P, _P, _P, _P, _P, _P, _I64, ctypes.POINTER(_I64)]),
    ("chapsim_props_train", _I, [_P, _I, ctypes.c_uint64, _I, _D, _DP]),
    ("chapsim_props_gate", _I, [_P, _D, _I, ctypes.POINTER(_I), _DP]),
    ("chapsim_set_props_mode", _I, [_P, _I, _P]),
    ("chapsim_therm_prop_update", _I, [_P, _I, _I]),
    ("chapsim_props_gate_outputs", _I, [_P, ctypes.POINTER(_I), _DP, _I]),
    ("chapsim_props_get_params", _I, [_P, _P, _I, _P, _I]),
    ("chapsim_props_set_params", _I, [_P, _P, _I, _P, _I]),
    ("chapsim_props_loss_grad", _I, [_P, _P, _P, _I, _DP, _P, _I]),
]
SIGNATURES += [
    ("chapsim_batch_create", _I, [ctypes.POINTER(ChapsimConfig), _I, ctypes.POINTER(_P)]),
    ("chapsim_batch_destroy", _I, [_P]),
    ("chapsim_batch_last_error", ctypes.c_char_p, [_P]),
    ("chapsim_batch_channel", _I, [_P, _I, ctypes.POINTER(_P)]),
    ("chapsim_batch_init_random", _I, [_P, ctypes.c_uint64, _D, _I]),
    ("chapsim_batch_autotune", _I, [_P, _I]),
    ("chapsim_batch_step", _I, [_P, _I]),
    ("chapsim_batch_sync", _I, [_P]),
    ("chapsim_batch_get_stream", _I, [_P, ctypes.POINTER(_P)]),
    ("chapsim_batch_kernels_per_step", _I, [_P, ctypes.POINTER(_I64)]),
]
SIGNATURES += [
    ("chapsim_divmax_noalloc", _I, [_P, _P, _P, _P, _I, _I, _I, _D, _D, _P, _P]),
]
SIGNATURES += [
    ("chapsim_io_config_default", _I, [ctypes.POINTER(ChapsimIOConfig)]),
    ("chapsim_create_io", _I, [ctypes.POINTER(ChapsimConfig), ctypes.POINTER(ChapsimIOConfig), ctypes.POINTER(_P)]),
    ("chapsim_set_table", _I, [_P, _P, _P, _P, _P, _P, _I, _I]),
    ("chapsim_rk3_eng_io", _I, [_P, _I]),
    ("chapsim_rk3_mom_io", _I, [_P, _I]),
    ("chapsim_step_io", _I, [_P, _I]),
    ("chapsim_io_set_inlet", _I, [_P, _P]),
    ("chapsim_step_coupled", _I, [_P, _P, _I]),
    ("chapsim_set_dt", _I, [_P, _D]),
    ("chapsim_stats", _I, [_P, _I]),
    ("chapsim_get_stats", _I, [_P, _I, _P, _I64, ctypes.POINTER(_I64)]),
    ("chapsim_stats_reset", _I, [_P]),
    ("chapsim_write_instant", _I, [_P, ctypes.c_char_p, _I, _D]),
    ("chapsim_read_instant", _I, [_P, ctypes.c_char_p, _D, ctypes.POINTER(_I), _DP]),
    ("chapsim_set_refinement", _I, [_P, _I]),
    ("chapsim_inject_wait_timeout", _I, [_P, _I]),
    ("chapsim_instant_file_name", _I, [ctypes.c_char_p, _I, ctypes.c_char_p, _D, ctypes.c_char_p, _I]),
    ("chapsim_instant_file_write", _I, [ctypes.c_char_p, _I, _I, _I, _I, _D, _D, _D, _P]),
    ("chapsim_instant_file_read", _I, [ctypes.c_char_p, _I, _I, _I, ctypes.POINTER(_I), _DP, _DP, _DP, _P]),
]
STATS_NV = 122
STATS_IO_NV = 360
PROPS_TABLE, PROPS_MLP = 0, 1
ERR_RANGE = 8
ERRORS[8] = "CHAPSIM_ERR_RANGE"
ERRORS[9] = "CHAPSIM_ERR_TOO_LARGE"
ERR_TOO_LARGE = 9

_lib = None


def load():
    """Load libchapsim.so once; raise if it is missing (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libchapsim.so not found at {LIB_PATH}; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C chapsim1ww_b200/csrc`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
