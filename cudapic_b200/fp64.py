"""All-FP64 twin of a discharge for the precision study
(``cudapic_fp64_*`` in include/cudapic.h).

The reference's launch sequence (Rust-CUDA/src/main.rs:1725-1808) with the
particles, fields, densities, collision tests and scattering in double: the
"all-FP64 GPU path" that the precision study sets beside the f32 paths and
eduPIC's FP64 CPU code.  A twin starts from a ``GpuSimState`` at the start of
an ion cycle (particles widened to double, the RNG planes copied, the RF phase
continued) and leaves the state unchanged.
"""
import ctypes as C

import numpy as np

from . import check, lib

E_CHARGE = 1.60217662e-19


class Fp64Discharge:
    def __init__(self, state):
        h = C.c_void_p()
        check(lib.cudapic_fp64_create(state.handle, C.byref(h)))
        self._h = h
        self.state = state
        self.params = state.params

    def close(self):
        if getattr(self, "_h", None):
            lib.cudapic_fp64_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()

    def run_steps(self, n):
        check(lib.cudapic_fp64_run_steps(self._h, int(n)))

    def run_cycles(self, n):
        self.run_steps(int(n) * self.params.n_t)

    def set_measure(self, on):
        check(lib.cudapic_fp64_set_measure(self._h, 1 if on else 0))

    def measurements(self):
        """Window sums (see cudapic_fp64_measurements) and derived figures:
        time-averaged densities, potential, the EEPF counts, the <j E> power
        [W/m^3], counts and the device error word."""
        n_g = self.params.n_g
        ce, ci, ps = (np.zeros(n_g, np.float64) for _ in range(3))
        eepf = np.zeros(2000, np.uint32)
        power = C.c_double()
        steps = (C.c_uint64 * 2)()
        counts = (C.c_uint32 * 2)()
        err = C.c_uint32()
        check(lib.cudapic_fp64_measurements(self._h, ce.ctypes.data, ci.ctypes.data, ps.ctypes.data, eepf.ctypes.data,
                                            C.addressof(power), C.addressof(steps), C.addressof(counts),
                                            C.addressof(err)))
        p = self.params
        n_steps, n_ion = steps[0], steps[1]
        return {
            "cumul_e": ce, "cumul_i": ci, "pot_sum": ps, "eepf": eepf, "power_sum": power.value,
            "steps": n_steps, "ion_steps": n_ion, "counts": (counts[0], counts[1]), "device_error": err.value,
            "ne": ce / max(n_steps, 1), "ni": ci / max(n_ion, 1), "pot": ps / max(n_steps, 1),
            "power_e": -E_CHARGE * p.weight / p.electrode_area / p.gap * power.value / max(n_steps, 1),
        }
