"""ctypes declarations of libcudapic.so (include/cudapic.h).

The library is loaded from this package directory only (built in-tree by
``cudapic_b200.build``).  There is no fallback: if the library is missing or
fails to load, importing the package raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcudapic.so")

OK = 0
ERR_CUDA = 1
ERR_CAPACITY = 2
ERR_ARG = 3
ERR_TIMEOUT = 4
ERR_NOT_SUPPORTED = 5
ERR_STATE = 6

DEVERR_SPAWN_E = 0x1
DEVERR_SPAWN_I = 0x2
DEVERR_POSITION = 0x4
DEVERR_ACTIVE = 0x8
DEVERR_TIMEOUT = 0x10
DEVERR_RECORDS = 0x20

FLAG_POISSON_F32_SCAN = 0x1
FLAG_DEPOSIT_FIXED_POINT = 0x2
FLAG_DEPOSIT_F32 = 0x4
CS_RANGES = 1_000_000
N_EEPF = 2000
ELECTRONS = 0
IONS = 1


class CudapicError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("cudapic status %d: %s" % (status, message))
        self.status = status


class Params(C.Structure):
    _fields_ = [
        ("n_g", C.c_uint32), ("n_t", C.c_uint32), ("n_sub", C.c_uint32), ("capacity", C.c_uint32),
        ("frequency", C.c_double), ("voltage", C.c_double), ("gap", C.c_double), ("pressure", C.c_double),
        ("temperature", C.c_double), ("weight", C.c_double), ("electrode_area", C.c_double),
        ("flags", C.c_uint32),
    ]


class Grid(C.Structure):
    _fields_ = [
        ("n_g", C.c_uint32), ("capacity", C.c_uint32), ("n_t", C.c_uint32), ("n_sub", C.c_uint32),
        ("flags", C.c_uint32),
        ("inv_dx", C.c_float), ("weight_factor", C.c_float), ("gap", C.c_float), ("dt_e", C.c_float),
        ("dt_i", C.c_float), ("factor_e", C.c_float), ("factor_i", C.c_float), ("e_charge", C.c_float),
        ("alpha", C.c_float), ("half_dx_over_eps", C.c_float), ("half_inv_dx", C.c_float),
        ("normal_range", C.c_float), ("f1", C.c_float), ("f2", C.c_float), ("half_me_over_e", C.c_float),
        ("half_mu_over_e", C.c_float), ("min_x", C.c_float), ("max_x", C.c_float),
        ("eepf_half_kick", C.c_float),
        ("dx", C.c_double), ("weight_factor_d", C.c_double), ("gas_density", C.c_double),
        ("voltage", C.c_double),
        ("dev_err", C.c_void_p), ("work", C.c_void_p), ("sigma_max_e", C.c_float),
    ]


class Tuning(C.Structure):
    _fields_ = [(name, C.c_int) for name in (
        "density_threads", "density_ctas_per_sm", "density_copies", "density_cluster",
        "push_stages", "push_ctas_per_sm", "mcc_stages", "mcc_ctas_per_sm", "mcc_variant", "step_stages",
        "step_ctas_per_sm", "step_rows", "inplace_ctas_per_sm", "inplace_copies", "inplace_prefetch",
        "scatter_ctas_per_sm")]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


N_IFED = 200


class WallCounters(C.Structure):
    """cudapic_wall_counters: particles absorbed at each electrode and the
    ion flux-energy distributions (1 eV bins)."""
    _fields_ = [("abs_pow", C.c_ulonglong), ("abs_gnd", C.c_ulonglong),
                ("ifed_pow", C.c_uint32 * N_IFED), ("ifed_gnd", C.c_uint32 * N_IFED)]

    def as_dict(self):
        import numpy as np
        return {"abs_pow": int(self.abs_pow), "abs_gnd": int(self.abs_gnd),
                "ifed_pow": np.array(self.ifed_pow, np.uint32), "ifed_gnd": np.array(self.ifed_gnd, np.uint32)}


class Precheck(C.Structure):
    """cudapic_precheck: the parameter-only accuracy conditions."""
    _fields_ = [("max_e_coll_dt_e", C.c_double), ("max_i_coll_dt_i", C.c_double), ("cfl_max_energy", C.c_double),
                ("conditions_ok", C.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Report(C.Structure):
    """cudapic_report: eduPIC's simulation report of a measurement window."""
    _fields_ = [("steps_measured", C.c_uint64)] + [(n, C.c_double) for n in (
        "density_center", "plasma_freq", "mean_energy_center", "debye_length", "e_coll_freq", "i_coll_freq",
        "wp_dt_e", "dx_over_debye", "max_e_coll_dt_e", "max_i_coll_dt_i")] + [("conditions_ok", C.c_int)] + [
        (n, C.c_double) for n in ("cfl_max_energy", "ion_flux_pow", "ion_flux_gnd", "mean_ion_energy_pow",
                                  "mean_ion_energy_gnd", "e_flux_pow", "e_flux_gnd", "power_e", "power_i")]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_P2 = C.c_void_p * 2


class Buffers(C.Structure):
    _fields_ = [
        ("x", _P2), ("vx", _P2), ("vy", _P2), ("vz", _P2),
        ("tmp_x", _P2), ("tmp_vx", _P2), ("tmp_vy", _P2), ("tmp_vz", _P2),
        ("rng", (C.c_void_p * 4) * 2),
        ("n_electrons", C.c_void_p), ("n_ions", C.c_void_p), ("alive_counter", C.c_void_p),
        ("efield", C.c_void_p), ("pot", C.c_void_p), ("e_density", C.c_void_p), ("i_density", C.c_void_p),
        ("cs", C.c_void_p), ("sigma_tot_e", C.c_void_p), ("sigma_tot_i", C.c_void_p),
        ("cumul_e_density", C.c_void_p), ("cumul_i_density", C.c_void_p), ("eepf", C.c_void_p),
        ("dev_err", C.c_void_p), ("work", C.c_void_p), ("sigma_max_e", C.c_float),
    ]


# (name, argtypes); every entry point returns int status unless noted.
_VP = C.c_void_p
_U32 = C.c_uint32
_F = C.c_float
_GP = C.POINTER(Grid)
SIGNATURES = {
    "cudapic_get_density": [_VP, _VP, _VP, _GP, _VP],
    "cudapic_solve_poisson_scan_f32": [_VP, _VP, _VP, _VP, _F, _GP, _VP],
    "cudapic_solve_poisson_dps_flexible": [_VP, _VP, _U32, _F, _F, _F, _VP],
    "cudapic_move_and_compact": [_VP] * 11 + [_F, _F, _GP, _VP],
    "cudapic_check_collisions_e": [_VP] * 17 + [_GP, _VP],
    "cudapic_check_collisions_i": [_VP] * 10 + [_GP, _VP],
    "cudapic_check_collisions_e_events": [_VP] * 18 + [_GP, _VP],
    "cudapic_check_collisions_e_deposit": [_VP] * 19 + [_GP, _VP],
    "cudapic_move_and_compact_deposit": [_VP] * 11 + [_F, _F, _VP, _GP, _VP],
    "cudapic_move_and_compact_wall": [_VP] * 11 + [_F, _F, _VP, C.c_int, _GP, _VP],
    "cudapic_state_wall_counters": [_VP, _VP],
    "cudapic_picdata_write": [C.c_char_p, C.c_double, _U32, _VP, _U32, _VP, _U32],
    "cudapic_picdata_read_header": [C.c_char_p, _VP, _VP, _VP, _VP],
    "cudapic_picdata_read": [C.c_char_p, _VP, _U32, _VP, _U32],
    "cudapic_state_save": [_VP, C.c_char_p],
    "cudapic_stability_precheck": [_VP, _VP],
    "cudapic_state_report": [_VP, _VP],
    "cudapic_state_write_info": [_VP, C.c_char_p],
    "cudapic_state_load": [_VP, C.c_char_p],
    "cudapic_step_electrons": [_VP] * 15 + [_F] + [_VP] * 9 + [_GP, _VP],
    "cudapic_step_electrons_noalloc": [_VP] * 15 + [_F] + [_VP] * 8 + [_GP, _VP],
    "cudapic_step_electrons_inplace": [_VP] * 11 + [_F] + [_VP] * 4 + [_GP, _VP],
    "cudapic_scatter_colliders_e": [_VP] * 20 + [_GP, _VP],
    "cudapic_check_collisions_i_events": [_VP] * 11 + [_GP, _VP],
    "cudapic_check_collisions_i_bounded": [_VP] * 10 + [_F, _VP, _GP, _VP],
    "cudapic_accumulate_density": [_VP, _VP, _GP, _VP],
    "cudapic_accumulate_eepf": [_VP] * 7 + [_GP, _VP],
    "cudapic_xoshiro128p_test_wrapper": [_U32, _U32, _U32, _U32, _VP, _VP],
    "cudapic_xoshiro128_seed_streams": [C.POINTER(_U32), _U32, _VP, _VP, _VP, _VP, _VP],
    "cudapic_cross_sections": [C.c_double, _VP, _VP, _VP],
    "cudapic_math_eval": [C.c_int, _VP, _VP, _VP, _U32, _VP],
    "cudapic_grid_from_params": [C.POINTER(Params), _GP],
    "cudapic_get_tuning": [C.POINTER(Tuning)],
    "cudapic_set_tuning": [C.POINTER(Tuning)],
    "cudapic_version": [],
    "cudapic_state_create": [C.POINTER(Params), C.c_int, C.POINTER(_VP)],
    "cudapic_state_destroy": [_VP],
    "cudapic_state_set_stream": [_VP, _VP],
    "cudapic_state_grid": [_VP, _GP],
    "cudapic_state_buffers": [_VP, C.POINTER(Buffers)],
    "cudapic_state_upload": [_VP, C.c_int, _VP, _VP, _VP, _VP, _U32],
    "cudapic_state_download": [_VP, C.c_int, _VP, _VP, _VP, _VP, _U32, C.POINTER(_U32)],
    "cudapic_state_seed": [_VP, C.POINTER(_U32), C.POINTER(_U32)],
    "cudapic_state_set_measure": [_VP, C.c_int],
    "cudapic_state_set_fused": [_VP, C.c_int],
    "cudapic_state_set_inplace": [_VP, C.c_int],
    "cudapic_state_set_spawn_collide": [_VP, C.c_int],
    "cudapic_state_set_solve_ahead": [_VP, C.c_int],
    "cudapic_state_set_overlap": [_VP, C.c_int],
    "cudapic_state_set_graphs": [_VP, C.c_int],
    "cudapic_state_run_steps": [_VP, C.c_uint64],
    "cudapic_state_counts": [_VP, C.POINTER(_U32), C.POINTER(_U32)],
    "cudapic_state_device_error": [_VP, C.POINTER(_U32)],
    "cudapic_state_debug_wait_timeout": [_VP, C.c_longlong],
    "cudapic_state_clear_device_error": [_VP],
    "cudapic_state_work": [_VP, C.POINTER(C.c_ulonglong)],
    "cudapic_state_steps_done": [_VP, C.POINTER(C.c_uint64)],
    "cudapic_state_synchronize": [_VP],
    "cudapic_state_download_measurements": [_VP, _VP, _VP, _VP],
    "cudapic_state_xt_shape": [_VP, C.POINTER(_U32), C.POINTER(_U32)],
    "cudapic_state_download_xt": [_VP, C.c_int, _VP],
    "cudapic_state_write_xt": [_VP, C.c_char_p],
    "cudapic_batch_create": [C.POINTER(_VP), _U32, C.POINTER(_VP)],
    "cudapic_batch_destroy": [_VP],
    "cudapic_batch_run_steps": [_VP, C.c_uint64],
    "cudapic_batch_synchronize": [_VP],
    "cudapic_batch_profile_steps": [_VP, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_uint64)],
    "cudapic_sens_create": [_VP, _U32, _U32, _U32, C.POINTER(_VP)],
    "cudapic_sens_forward": [_VP, C.c_double, C.POINTER(C.c_double)],
    "cudapic_sens_backward": [_VP, C.POINTER(C.c_double)],
    "cudapic_sens_info": [_VP, C.POINTER(_U32), C.POINTER(_U32), C.POINTER(C.c_uint64)],
    "cudapic_sens_download": [_VP, C.c_int, _VP, _VP, _VP, _VP, _VP, _U32],
    "cudapic_sens_destroy": [_VP],
    "cudapic_fp64_create": [_VP, C.POINTER(_VP)],
    "cudapic_fp64_set_measure": [_VP, C.c_int],
    "cudapic_fp64_run_steps": [_VP, C.c_uint64],
    "cudapic_fp64_measurements": [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP],
    "cudapic_fp64_destroy": [_VP],
}
OTHER = {
    "cudapic_params_default": (None, [C.POINTER(Params)]),
    "cudapic_status_string": (C.c_char_p, [C.c_int]),
    "cudapic_last_error": (C.c_char_p, []),
    "cudapic_state_stream": (_VP, [_VP]),
    "cudapic_batch_stream": (_VP, [_VP]),
}


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError("libcudapic.so not found at %s: build it with `python -m cudapic_b200.build` "
                          "(there is no CPU fallback)" % path)
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    for name, (res, args) in OTHER.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


def exported_symbols():
    return sorted(list(SIGNATURES) + list(OTHER))
