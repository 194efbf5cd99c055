"""Simulation state and per-step driver (host mirror of GpuSimState).

``GpuSimState`` wraps ``cudapic_state`` (include/cudapic.h), the B200
counterpart of the reference's GpuSimState (Rust-CUDA/src/main.rs:131-350):
SoA f32 particle buffers preallocated to ``capacity`` per species, device
counters, per-slot xoshiro128+ planes, cross-section tables and measurement
accumulators.  ``run_steps`` enqueues the reference's per-step loop
(Rust-CUDA/src/main.rs:1728-1807) replayed from CUDA graphs.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib, check, default_params, lib

# master seeds of the reference driver, Rust-CUDA/src/main.rs:1666-1673
E_MASTER_SEED = (0x12345678, 0x11112222, 0x22223333, 0x33334444)
I_MASTER_SEED = (0x44445555, 0x55556666, 0x66667777, 0x77778888)


@dataclass
class ParticlesSoA:
    """Host particle container (Rust-CUDA/src/main.rs:112-129)."""
    x: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray

    @classmethod
    def with_capacity(cls, cap):
        return cls(*(np.zeros(cap, np.float32) for _ in range(4)))

    def __len__(self):
        return len(self.x)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class GpuSimState:
    """Owns every device buffer of one discharge on one GPU."""

    def __init__(self, params=None, device=0, **overrides):
        if params is None:
            params = default_params(**overrides)
        self.params = params
        self.device = device
        h = C.c_void_p()
        check(lib.cudapic_state_create(C.byref(params), int(device), C.byref(h)))
        self._h = h
        self.grid = _lib.Grid()
        check(lib.cudapic_state_grid(self._h, C.byref(self.grid)))
        self.capacity = self.grid.capacity
        self.fused = True

    # -- lifetime -----------------------------------------------------
    @classmethod
    def allocate(cls, params=None, device=0, **overrides):
        """GpuSimState::allocate (Rust-CUDA/src/main.rs:187-250)."""
        return cls(params, device, **overrides)

    def close(self):
        if getattr(self, "_h", None):
            lib.cudapic_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def stream(self):
        return lib.cudapic_state_stream(self._h) or 0

    def set_stream(self, stream):
        s = stream if isinstance(stream, int) else stream.cuda_stream
        check(lib.cudapic_state_set_stream(self._h, s))

    def buffers(self):
        b = _lib.Buffers()
        check(lib.cudapic_state_buffers(self._h, C.byref(b)))
        return b

    # -- host <-> device (Rust-CUDA/src/main.rs:252-349) ---------------
    def _upload(self, species, x, vx, vy, vz):
        arrs = [_f32(a) for a in (x, vx, vy, vz)]
        n = len(arrs[0])
        check(lib.cudapic_state_upload(self._h, species, *(a.ctypes.data for a in arrs), n))

    def upload_electrons(self, particles, n_active=None):
        n = len(particles) if n_active is None else n_active
        self._upload(_lib.ELECTRONS, particles.x[:n], particles.vx[:n], particles.vy[:n], particles.vz[:n])

    def upload_ions(self, particles, n_active=None):
        n = len(particles) if n_active is None else n_active
        self._upload(_lib.IONS, particles.x[:n], particles.vx[:n], particles.vy[:n], particles.vz[:n])

    def _download(self, species):
        out = ParticlesSoA.with_capacity(self.capacity)
        n = C.c_uint32()
        check(lib.cudapic_state_download(self._h, species, out.x.ctypes.data, out.vx.ctypes.data,
                                         out.vy.ctypes.data, out.vz.ctypes.data, self.capacity, C.byref(n)))
        k = n.value
        return ParticlesSoA(out.x[:k].copy(), out.vx[:k].copy(), out.vy[:k].copy(), out.vz[:k].copy()), k

    def download_electrons(self):
        return self._download(_lib.ELECTRONS)

    def download_ions(self):
        return self._download(_lib.IONS)

    def seed(self, e_master=E_MASTER_SEED, i_master=I_MASTER_SEED):
        """xoshiro128_seed_streams for every slot of both species (on the GPU)."""
        em = (C.c_uint32 * 4)(*e_master)
        im = (C.c_uint32 * 4)(*i_master)
        check(lib.cudapic_state_seed(self._h, em, im))

    upload_rng_state = seed

    def set_measure(self, on=True):
        check(lib.cudapic_state_set_measure(self._h, 1 if on else 0))

    def set_fused(self, on=True):
        """Fused driver step: the electron kernel pushes, collides and deposits
        the next density in one launch (default on); off: the reference's
        launch sequence."""
        check(lib.cudapic_state_set_fused(self._h, 1 if on else 0))
        self.fused = bool(on)

    inplace = True   # the library's default

    def set_inplace(self, on=True):
        """Fused mode: in-place electron steps between compacting ones (default on)."""
        check(lib.cudapic_state_set_inplace(self._h, 1 if on else 0))
        self.inplace = bool(on)

    def set_spawn_collide(self, on=True):
        """eduPIC semantics: electrons born in a step are tested for collision
        in that step (in-place steps; default off, the GPU reference's)."""
        check(lib.cudapic_state_set_spawn_collide(self._h, 1 if on else 0))

    def set_solve_ahead(self, on=True):
        """In-place steps solve the next step's field in their scatter pass
        (default on) instead of in a Poisson kernel of the next step."""
        check(lib.cudapic_state_set_solve_ahead(self._h, 1 if on else 0))

    def set_graphs(self, on=True):
        """Replay captured CUDA graphs (default) or launch every step from the host."""
        check(lib.cudapic_state_set_graphs(self._h, 1 if on else 0))

    def set_overlap(self, on=True):
        """Programmatic dependent launch between the step's kernels (default on)."""
        check(lib.cudapic_state_set_overlap(self._h, 1 if on else 0))

    def save(self, path):
        """Checkpoint in eduPIC's picdata.bin format (plus ``path``.rng)."""
        check(lib.cudapic_state_save(self._h, str(path).encode()))

    def load(self, path):
        """Resume from a picdata.bin (this library's or eduPIC's)."""
        check(lib.cudapic_state_load(self._h, str(path).encode()))

    def report(self):
        """eduPIC's simulation report of the measurement window (dict)."""
        r = _lib.Report()
        check(lib.cudapic_state_report(self._h, C.byref(r)))
        return r.as_dict()

    def write_info(self, path):
        """The report as eduPIC's info.txt."""
        check(lib.cudapic_state_write_info(self._h, str(path).encode()))

    def xt_shape(self):
        """(n_g, n_xt) of the XT diagnostics; n_xt = 0 without them."""
        n_g, n_xt = C.c_uint32(), C.c_uint32()
        check(lib.cudapic_state_xt_shape(self._h, C.byref(n_g), C.byref(n_xt)))
        return n_g.value, n_xt.value

    def download_xt(self, quantity):
        """One normalised XT quantity of the measurement window (name of
        XT_NAMES or its index) as an [n_g, n_xt] array (eduPIC's *_xt.dat)."""
        q = XT_NAMES.index(quantity) if isinstance(quantity, str) else int(quantity)
        n_g, n_xt = self.xt_shape()
        out = np.zeros((n_g, n_xt), np.float64)
        check(lib.cudapic_state_download_xt(self._h, q, out.ctypes.data))
        return out

    def write_xt(self, directory):
        """eduPIC's eleven *_xt.dat files in `directory`."""
        check(lib.cudapic_state_write_xt(self._h, str(directory).encode()))

    def wall_counters(self):
        """Electrode counters of the measurement window:
        {"e": {...}, "i": {...}} with abs_pow, abs_gnd, ifed_pow, ifed_gnd."""
        out = (_lib.WallCounters * 2)()
        check(lib.cudapic_state_wall_counters(self._h, out))
        return {"e": out[0].as_dict(), "i": out[1].as_dict()}

    def download_measurements(self):
        n_g = self.grid.n_g
        ce = np.zeros(n_g, np.float64)
        ci = np.zeros(n_g, np.float64)
        eepf = np.zeros(_lib.N_EEPF, np.uint32)
        check(lib.cudapic_state_download_measurements(self._h, ce.ctypes.data, ci.ctypes.data, eepf.ctypes.data))
        return ce, ci, eepf

    # -- stepping -------------------------------------------------------
    def run_steps(self, n_steps):
        check(lib.cudapic_state_run_steps(self._h, int(n_steps)))

    def run_cycles(self, n_cycles):
        self.run_steps(int(n_cycles) * self.params.n_t)

    def counts(self):
        ne, ni = C.c_uint32(), C.c_uint32()
        check(lib.cudapic_state_counts(self._h, C.byref(ne), C.byref(ni)))
        return ne.value, ni.value

    def device_error(self, raise_on_error=False):
        bits = C.c_uint32()
        rc = lib.cudapic_state_device_error(self._h, C.byref(bits))
        if raise_on_error:
            check(rc)
        elif rc not in (_lib.OK, _lib.ERR_CAPACITY, _lib.ERR_TIMEOUT):
            check(rc)
        return bits.value

    def clear_device_error(self):
        check(lib.cudapic_state_clear_device_error(self._h))

    def work(self):
        w = C.c_ulonglong()
        check(lib.cudapic_state_work(self._h, C.byref(w)))
        return w.value

    def steps_done(self):
        s = C.c_uint64()
        check(lib.cudapic_state_steps_done(self._h, C.byref(s)))
        return s.value

    def synchronize(self):
        check(lib.cudapic_state_synchronize(self._h))


# XT quantities in the order of eduPIC's save_all_xt files (CUDAPIC_XT_*)
XT_NAMES = ("pot", "efield", "ne", "ni", "je", "ji", "powere", "poweri", "meanee", "meanei", "ioniz")


class GpuBatch:
    """Discharges (GpuSimState objects on one device) stepped in lockstep:
    every kernel of a step is one launch over all of them
    (cudapic_batch_*).  The states keep their buffers and API; close the
    batch before the states."""

    def __init__(self, states):
        self.states = list(states)
        arr = (C.c_void_p * len(self.states))(*[st.handle for st in self.states])
        h = C.c_void_p()
        check(lib.cudapic_batch_create(arr, len(self.states), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.cudapic_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self):
        return lib.cudapic_batch_stream(self._h) or 0

    def run_steps(self, n_steps):
        check(lib.cudapic_batch_run_steps(self._h, int(n_steps)))

    @property
    def inplace(self):
        """True when the batch's electron steps run in place between compacting ones."""
        return all(st.inplace for st in self.states)

    BATCH_KERNELS = ("poisson", "ion_push", "electron_step", "ion_collisions", "electron_inplace",
                     "electron_scatter")

    def profile_steps(self, n_steps):
        """Runs n_steps uncaptured with CUDA events around every kernel
        (cudapic_batch_profile_steps); returns {kernel: (ms summed, launches)}."""
        ms = (C.c_double * len(self.BATCH_KERNELS))()
        n = (C.c_uint64 * len(self.BATCH_KERNELS))()
        check(lib.cudapic_batch_profile_steps(self._h, int(n_steps), ms, n))
        return {k: (ms[j], n[j]) for j, k in enumerate(self.BATCH_KERNELS)}

    def run_cycles(self, n_cycles):
        self.run_steps(int(n_cycles) * self.states[0].params.n_t)

    def synchronize(self):
        check(lib.cudapic_batch_synchronize(self._h))
