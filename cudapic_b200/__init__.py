"""cudapic_b200: B200-native (sm_100a) PIC/MCC cycle of cudaPIC.

The compute lives in ``libcudapic.so`` (hand-written CUDA behind a C ABI,
``include/cudapic.h``).  This package is a thin host mirror of the
reference's interfaces:

* ``cudapic_b200.kernels`` -- one function per reference kernel
  (``get_density``, ``solve_poisson_scan_f32``, ``move_and_compact``,
  ``check_collisions_e``, ``check_collisions_i``, ``accumulate_density``,
  ``accumulate_eepf``, ``xoshiro128p_test_wrapper``,
  ``solve_poisson_dps_flexible``) taking device tensors, as the cuda-oxide
  typed launchers of Rust-CUDA/src/main.rs:1705-1806 take device buffers;
* ``cudapic_b200.sim.GpuSimState`` -- the reference's GpuSimState
  (Rust-CUDA/src/main.rs:131-350) plus its per-step loop.

Importing the package loads the library; a missing library raises
ImportError (there is no CPU fallback).
"""
import ctypes as _C

from . import _lib
from ._lib import (CS_RANGES, ELECTRONS, IONS, N_EEPF, Buffers, CudapicError, Grid, Params,  # noqa: F401
                   FLAG_POISSON_F32_SCAN, FLAG_DEPOSIT_FIXED_POINT, FLAG_DEPOSIT_F32, DEVERR_SPAWN_E, DEVERR_SPAWN_I, DEVERR_POSITION,
                   DEVERR_ACTIVE, DEVERR_TIMEOUT)

lib = _lib.load()
LIB_PATH = _lib.LIB_PATH


def check(status):
    """Raise CudapicError for a non-zero status of an entry point."""
    if status != _lib.OK:
        msg = lib.cudapic_last_error()
        raise CudapicError(status, msg.decode() if msg else lib.cudapic_status_string(status).decode())
    return status


def default_params(**overrides):
    """Reference constants (Rust-CUDA/src/main.rs:40-50, :79) with overrides."""
    p = Params()
    lib.cudapic_params_default(_C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError("unknown parameter %r" % k)
        setattr(p, k, v)
    return p


def grid_from_params(params=None, **overrides):
    if params is None:
        params = default_params(**overrides)
    g = Grid()
    check(lib.cudapic_grid_from_params(_C.byref(params), _C.byref(g)))
    return g


def version():
    return lib.cudapic_version()


def get_tuning():
    """Current kernel launch shapes (cudapic_tuning) as a dict."""
    t = _lib.Tuning()
    check(lib.cudapic_get_tuning(_C.byref(t)))
    return t.as_dict()


def set_tuning(**fields):
    """Updates kernel launch shapes; unspecified fields keep their values."""
    cur = get_tuning()
    for k, v in fields.items():
        if k not in cur:
            raise AttributeError("unknown tuning field %r" % k)
        cur[k] = int(v)
    t = _lib.Tuning(**cur)
    check(lib.cudapic_set_tuning(_C.byref(t)))
    return get_tuning()


def stability_precheck(params=None, **overrides):
    """The accuracy conditions that follow from the parameters alone
    (cudapic_stability_precheck): max collision frequency x time step for
    electrons and ions, and the CFL energy limit."""
    p = params if params is not None else default_params(**overrides)
    out = _lib.Precheck()
    check(lib.cudapic_stability_precheck(_C.byref(p), _C.byref(out)))
    return out.as_dict()


from . import kernels  # noqa: E402,F401
from . import sim  # noqa: E402,F401
