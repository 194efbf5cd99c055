"""CPU tests of the C-ABI library: it loads, exports every entry point that
include/cudapic.h declares, and its host-side logic (derived constants,
cross-section tables, argument validation) agrees with the oracle.  No
kernel is launched."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cudapic.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cudapic_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(cudapic):
    declared = _declared_functions()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", cudapic.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s(cudapic_[a-z0-9_]+)$", out, flags=re.M))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    for f in declared:
        getattr(cudapic.lib, f)  # resolvable through ctypes


def test_python_bindings_cover_header(cudapic):
    from cudapic_b200 import _lib
    assert set(_declared_functions()) == set(_lib.exported_symbols())


def test_version(cudapic):
    assert cudapic.version() == 100


def test_grid_matches_oracle_constants(cudapic, oracle):
    for n_g, v, p, gap in [(400, 250.0, 10.0, 0.025), (4096, 250.0, 10.0, 0.025), (200, 137.5, 31.0, 0.0173)]:
        g = cudapic.grid_from_params(n_g=n_g, voltage=v, pressure=p, gap=gap)
        ph = oracle.phys_from_params(n_g=n_g, voltage=v, pressure=p, gap=gap)
        for name in ("inv_dx", "weight_factor", "gap", "dt_e", "dt_i", "factor_e", "factor_i", "e_charge", "alpha",
                     "half_dx_over_eps", "half_inv_dx", "normal_range", "f1", "f2", "half_me_over_e",
                     "half_mu_over_e", "min_x", "max_x", "eepf_half_kick", "dx", "weight_factor_d",
                     "gas_density"):
            assert getattr(g, name) == getattr(ph, name), name


def test_cross_sections_bit_exact_with_oracle(cudapic, oracle, tables):
    cs, se, si = cudapic.kernels.init_cross_sections(oracle.phys_from_params().gas_density)
    ocs, ose, osi = tables
    assert np.array_equal(cs.view(np.uint32), ocs.view(np.uint32))
    assert np.array_equal(se.view(np.uint32), ose.view(np.uint32))
    assert np.array_equal(si.view(np.uint32), osi.view(np.uint32))
    # thresholds: no excitation below 11.5 eV, no ionization below 15.8 eV
    assert cs[1_000_000 + 11500] == 0 and cs[1_000_000 + 11501] > 0
    assert cs[2_000_000 + 15800] == 0 and cs[2_000_000 + 15801] > 0


def test_argument_validation_without_device(cudapic):
    from cudapic_b200 import _lib
    g = cudapic.grid_from_params()
    lib = cudapic.lib
    assert lib.cudapic_get_density(None, None, None, C.byref(g), None) == _lib.ERR_ARG
    assert lib.cudapic_move_and_compact(*([None] * 11), C.c_float(1.0), C.c_float(1.0), C.byref(g), None) == _lib.ERR_ARG
    bad = cudapic.grid_from_params()
    bad.n_g = 2
    assert lib.cudapic_get_density(1, 2, 3, C.byref(bad), None) == _lib.ERR_ARG
    assert b"n_g" in lib.cudapic_last_error()
    zero = (C.c_uint32 * 4)(0, 0, 0, 0)
    assert lib.cudapic_xoshiro128_seed_streams(zero, 4, 1, 2, 3, 4, None) == _lib.ERR_ARG
    with pytest.raises(cudapic.CudapicError):
        cudapic.grid_from_params(n_g=1)
    with pytest.raises(cudapic.CudapicError):
        cudapic.grid_from_params(capacity=0)
    # the no-alloc fused step: checks come before any device work
    ptrs = list(range(256, 256 + 16 * 15, 16))
    tail = list(range(4096, 4096 + 16 * 8, 16))
    assert lib.cudapic_step_electrons_noalloc(*ptrs, C.c_float(1.0), *tail[:4], None, *tail[5:], C.byref(g),
                                              None) == _lib.ERR_ARG
    big = cudapic.grid_from_params()
    big.capacity = 0x80000004
    assert lib.cudapic_step_electrons_noalloc(*ptrs, C.c_float(1.0), *tail, C.byref(big), None) == _lib.ERR_ARG
    assert b"CUDAPIC_NOALLOC_MAX_CAPACITY" in lib.cudapic_last_error()
    # sensitivity and FP64-twin objects: null handles are refused, destroy(NULL) is a no-op
    h = C.c_void_p()
    assert lib.cudapic_sens_create(None, 8000, 200, 0, C.byref(h)) == _lib.ERR_ARG
    out2 = (C.c_double * 2)()
    assert lib.cudapic_sens_forward(None, C.c_double(250.0), out2) == _lib.ERR_ARG
    assert lib.cudapic_sens_backward(None, out2) == _lib.ERR_ARG
    assert lib.cudapic_sens_destroy(None) == _lib.OK
    assert lib.cudapic_fp64_create(None, C.byref(h)) == _lib.ERR_ARG
    assert lib.cudapic_fp64_run_steps(None, 1) == _lib.ERR_ARG
    assert lib.cudapic_fp64_destroy(None) == _lib.OK


def test_state_create_reports_missing_device(cudapic):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(cudapic.CudapicError) as ei:
        cudapic.sim.GpuSimState(capacity=1024)
    assert ei.value.status in (1, 5)
