"""eduPIC's particle checkpoint file picdata.bin through libcudapic's C ABI.

The format is eduPIC's own (save_particle_data / load_particle_data,
C/eduPIC.cc:726-781): doubles [Time, cycles_done, N_e, x_e..., vx_e...,
vy_e..., vz_e..., N_i, x_i..., ...].  These helpers work on host arrays and
need no GPU; ``GpuSimState.save`` / ``.load`` checkpoint a running discharge
(particles plus the RNG planes in ``<path>.rng``).
"""
import ctypes as C

import numpy as np

from . import check, lib


def _planes(arrays):
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in arrays]
    return arrs, (C.c_void_p * 4)(*[a.ctypes.data for a in arrs])


def write_picdata(path, electrons, ions, time=0.0, cycles_done=0):
    """electrons / ions: (x, vx, vy, vz) arrays of one species each."""
    e, ep = _planes(electrons)
    i, ip = _planes(ions)
    check(lib.cudapic_picdata_write(str(path).encode(), float(time), int(cycles_done), ep, len(e[0]), ip,
                                    len(i[0])))


def read_picdata(path):
    """Returns (time, cycles_done, electrons, ions), each species a tuple of
    four float32 arrays (the file's doubles rounded to f32)."""
    t, cyc, ne, ni = C.c_double(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    check(lib.cudapic_picdata_read_header(str(path).encode(), C.byref(t), C.byref(cyc), C.byref(ne), C.byref(ni)))
    e = [np.empty(max(ne.value, 1), np.float32) for _ in range(4)]
    i = [np.empty(max(ni.value, 1), np.float32) for _ in range(4)]
    ep = (C.c_void_p * 4)(*[a.ctypes.data for a in e])
    ip = (C.c_void_p * 4)(*[a.ctypes.data for a in i])
    check(lib.cudapic_picdata_read(str(path).encode(), ep, ne.value, ip, ni.value))
    return (t.value, cyc.value, tuple(a[:ne.value] for a in e), tuple(a[:ni.value] for a in i))
