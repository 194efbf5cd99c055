"""Reference-named launchers of the cudaPIC kernels.

Mirrors the cuda-oxide module ``kernels`` (Rust-CUDA/src/main.rs:352-1358):
same names, same argument order (device buffers, then scalars), plus the
runtime ``grid`` (the reference's compile-time constants) and an optional
``stream``.  Buffers are CUDA tensors (anything with ``data_ptr()``) or raw
device pointers (int).  Launches are asynchronous on ``stream`` (default:
torch's current stream when a tensor is passed, else the legacy default
stream).  A failing launch raises CudapicError, as the reference's launchers
return Err(DriverError) (:1730-1806).
"""
import ctypes as C

import numpy as np

from . import _lib, check, lib

__all__ = ["get_density", "solve_poisson_scan_f32", "solve_poisson_dps_flexible", "move_and_compact",
           "check_collisions_e", "check_collisions_i", "accumulate_density", "accumulate_eepf",
           "xoshiro128p_test_wrapper", "xoshiro128_seed_streams", "init_cross_sections", "math_eval"]


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream(stream, *tensors):
    if stream is not None:
        return stream if isinstance(stream, int) else stream.cuda_stream
    for t in tensors:
        if hasattr(t, "is_cuda") and t.is_cuda:
            import torch
            return torch.cuda.current_stream(t.device).cuda_stream
    return 0


def _g(grid):
    return C.byref(grid)


def get_density(x, density, n_active, grid, stream=None):
    """get_density (Rust-CUDA/src/main.rs:356-406): adds the CIC deposit of
    x[0:n_active] to density (zero it first)."""
    check(lib.cudapic_get_density(_ptr(x), _ptr(density), _ptr(n_active), _g(grid), _stream(stream, x)))


def solve_poisson_scan_f32(e_density, i_density, pot, efield, pot0, grid, stream=None):
    """solve_poisson_scan_f32 (Rust-CUDA/src/main.rs:408-494)."""
    check(lib.cudapic_solve_poisson_scan_f32(_ptr(e_density), _ptr(i_density), _ptr(pot), _ptr(efield),
                                             float(pot0), _g(grid), _stream(stream, pot)))


def solve_poisson_dps_flexible(source, pot, n, psi_left, psi_right, dx, stream=None):
    """solve_poisson_dps_flexible (Rust-CUDA/src/main.rs:496-564)."""
    check(lib.cudapic_solve_poisson_dps_flexible(_ptr(source), _ptr(pot), int(n), float(psi_left),
                                                 float(psi_right), float(dx), _stream(stream, pot)))


def move_and_compact(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, alive_counter,
                     n_active, factor, dt, grid, stream=None):
    """move_and_compact (Rust-CUDA/src/main.rs:566-678)."""
    check(lib.cudapic_move_and_compact(_ptr(efield), _ptr(src_x), _ptr(src_vx), _ptr(src_vy), _ptr(src_vz),
                                       _ptr(dst_x), _ptr(dst_vx), _ptr(dst_vy), _ptr(dst_vz),
                                       _ptr(alive_counter), _ptr(n_active), float(factor), float(dt), _g(grid),
                                       _stream(stream, src_x)))


def move_and_compact_deposit(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, alive_counter,
                             n_active, factor, dt, next_density, grid, stream=None):
    """move_and_compact fused with the deposit of the survivors' new
    positions into next_density (no reference counterpart)."""
    check(lib.cudapic_move_and_compact_deposit(_ptr(efield), _ptr(src_x), _ptr(src_vx), _ptr(src_vy),
                                               _ptr(src_vz), _ptr(dst_x), _ptr(dst_vx), _ptr(dst_vy), _ptr(dst_vz),
                                               _ptr(alive_counter), _ptr(n_active), float(factor), float(dt),
                                               _ptr(next_density), _g(grid), _stream(stream, src_x)))


def check_collisions_e_deposit(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                               i_vz, alive_e, alive_i, e_next_density, i_next_density, grid, stream=None):
    """check_collisions_e whose spawns are also deposited (no reference counterpart)."""
    args = [_ptr(a) for a in (total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                              i_vz, alive_e, alive_i, e_next_density, i_next_density)]
    check(lib.cudapic_check_collisions_e_deposit(*args, _g(grid), _stream(stream, vx)))


def move_and_compact_wall(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, alive_counter,
                          n_active, factor, dt, wall, ions, grid, stream=None):
    """move_and_compact that also counts the particles absorbed at each
    electrode into the device block `wall` (cudapic_wall_counters; ions also
    fill the IFEDs), the boundary check of C/eduPIC.cc:623-667."""
    check(lib.cudapic_move_and_compact_wall(_ptr(efield), _ptr(src_x), _ptr(src_vx), _ptr(src_vy), _ptr(src_vz),
                                            _ptr(dst_x), _ptr(dst_vx), _ptr(dst_vy), _ptr(dst_vz),
                                            _ptr(alive_counter), _ptr(n_active), float(factor), float(dt), _ptr(wall),
                                            1 if ions else 0, _g(grid), _stream(stream, src_x)))


def step_electrons(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, rng0, rng1, rng2, rng3,
                   total_cs_e, cs, sigma_max_e, i_x, i_vx, i_vy, i_vz, alive_counter, n_e, n_i, e_next_density,
                   i_next_density, grid, stream=None):
    """Fused electron step: push, collisions with the RNG stream of each
    electron's source slot, compaction and next-step deposit in one launch
    (does the work of move_and_compact + check_collisions_e + get_density)."""
    head = [_ptr(a) for a in (efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, rng0, rng1, rng2,
                              rng3, total_cs_e, cs)]
    tail = [_ptr(a) for a in (i_x, i_vx, i_vy, i_vz, alive_counter, n_e, n_i, e_next_density, i_next_density)]
    check(lib.cudapic_step_electrons(*head, float(sigma_max_e), *tail, _g(grid), _stream(stream, src_x)))


def step_electrons_noalloc(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, rng0, rng1, rng2,
                           rng3, total_cs_e, cs, sigma_max_e, i_x, i_vx, i_vy, i_vz, n_e, n_i, e_next_density,
                           i_next_density, grid, stream=None):
    """step_electrons for callers that cannot allocate device memory: no
    slot counter is passed (the library keeps it in a static device array)
    and the new electron count is written into n_e in place."""
    head = [_ptr(a) for a in (efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, rng0, rng1, rng2,
                              rng3, total_cs_e, cs)]
    tail = [_ptr(a) for a in (i_x, i_vx, i_vy, i_vz, n_e, n_i, e_next_density, i_next_density)]
    check(lib.cudapic_step_electrons_noalloc(*head, float(sigma_max_e), *tail, _g(grid), _stream(stream, src_x)))


def _planes8(coll):
    """The eight collider-record planes as a C array of device pointers."""
    import ctypes
    if len(coll) != 8:
        raise ValueError("eight record planes: slot, vx, vy, vz, rng0..3")
    return (ctypes.c_void_p * 8)(*[_ptr(a) for a in coll])


def step_electrons_inplace(efield, x, vx, vy, vz, rng0, rng1, rng2, rng3, total_cs_e, cs, sigma_max_e, n_e, coll,
                           n_colliders, e_next_density, grid, stream=None):
    """In-place electron step, stream pass: push, absorption (x set to
    CUDAPIC_DEAD_X), collision test and next-step deposit with every electron
    kept in its slot; each collider recorded in the eight `coll` planes
    (slot, vx, vy, vz, RNG state), its slot's RNG state advanced past its
    scattering's draws."""
    head = [_ptr(a) for a in (efield, x, vx, vy, vz, rng0, rng1, rng2, rng3, total_cs_e, cs)]
    check(lib.cudapic_step_electrons_inplace(*head, float(sigma_max_e), _ptr(n_e), _planes8(coll), _ptr(n_colliders),
                                             _ptr(e_next_density), _g(grid), _stream(stream, x)))


def scatter_colliders_e(x, vx, vy, vz, rng0, rng1, rng2, rng3, cs, coll, n_colliders, ticket, i_x, i_vx, i_vy,
                        i_vz, n_e, n_i, e_next_density, i_next_density, grid, stream=None):
    """In-place electron step, scatter pass over the recorded colliders
    (spawns appended at n_e and n_i)."""
    head = [_ptr(a) for a in (x, vx, vy, vz, rng0, rng1, rng2, rng3, cs)]
    tail = [_ptr(a) for a in (n_colliders, ticket, i_x, i_vx, i_vy, i_vz, n_e, n_i, e_next_density, i_next_density)]
    check(lib.cudapic_scatter_colliders_e(*head, _planes8(coll), *tail, _g(grid), _stream(stream, x)))


def check_collisions_e(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy, i_vz,
                       alive_e, alive_i, grid, stream=None, events=None):
    """check_collisions_e (Rust-CUDA/src/main.rs:971-1165).  With `events`
    (uint8 buffer), also records each particle's collision type."""
    args = [_ptr(a) for a in (total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                              i_vz, alive_e, alive_i)]
    s = _stream(stream, vx)
    if events is None:
        check(lib.cudapic_check_collisions_e(*args, _g(grid), s))
    else:
        check(lib.cudapic_check_collisions_e_events(*args, _ptr(events), _g(grid), s))


def check_collisions_i(total_cs_i, cs, active_i, vx, vy, vz, rng0, rng1, rng2, rng3, grid, stream=None,
                       events=None, sigma_max_i=None):
    """check_collisions_i (Rust-CUDA/src/main.rs:1167-1292).  sigma_max_i
    (the largest entry of total_cs_i): the bounded entry, same results."""
    args = [_ptr(a) for a in (total_cs_i, cs, active_i, vx, vy, vz, rng0, rng1, rng2, rng3)]
    s = _stream(stream, vx)
    if sigma_max_i is not None:
        check(lib.cudapic_check_collisions_i_bounded(*args, float(sigma_max_i), _ptr(events) if events is not None
                                                     else None, _g(grid), s))
    elif events is None:
        check(lib.cudapic_check_collisions_i(*args, _g(grid), s))
    else:
        check(lib.cudapic_check_collisions_i_events(*args, _ptr(events), _g(grid), s))


def accumulate_density(density, cumul, grid, stream=None):
    """accumulate_density (Rust-CUDA/src/main.rs:1294-1299)."""
    check(lib.cudapic_accumulate_density(_ptr(density), _ptr(cumul), _g(grid), _stream(stream, density)))


def accumulate_eepf(x, vx, vy, vz, efield, active_e, eepf, grid, stream=None):
    """accumulate_eepf (Rust-CUDA/src/main.rs:1301-1339)."""
    check(lib.cudapic_accumulate_eepf(_ptr(x), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(efield), _ptr(active_e),
                                      _ptr(eepf), _g(grid), _stream(stream, x)))


def xoshiro128p_test_wrapper(s0, s1, s2, s3, dest, stream=None):
    """xoshiro128p_test_wrapper (Rust-CUDA/src/main.rs:1341-1357)."""
    check(lib.cudapic_xoshiro128p_test_wrapper(s0, s1, s2, s3, _ptr(dest), _stream(stream, dest)))


def xoshiro128_seed_streams(master, n, rng0, rng1, rng2, rng3, stream=None):
    """xoshiro128_seed_streams (Rust-CUDA/src/main.rs:1446-1496) on the GPU."""
    m = (C.c_uint32 * 4)(*[int(v) & 0xFFFFFFFF for v in master])
    check(lib.cudapic_xoshiro128_seed_streams(m, int(n), _ptr(rng0), _ptr(rng1), _ptr(rng2), _ptr(rng3),
                                              _stream(stream, rng0)))


def init_cross_sections(gas_density):
    """init_cross_sections (Rust-CUDA/src/main.rs:1378-1444), host: returns
    numpy (cs[5*1e6], sigma_tot_e[1e6], sigma_tot_i[1e6])."""
    cs = np.empty(5 * _lib.CS_RANGES, np.float32)
    se = np.empty(_lib.CS_RANGES, np.float32)
    si = np.empty(_lib.CS_RANGES, np.float32)
    check(lib.cudapic_cross_sections(float(gas_density), cs.ctypes.data, se.ctypes.data, si.ctypes.data))
    return cs, se, si


MATH_FN = {"exp": 0, "log": 1, "sin": 2, "cos": 3, "tan": 4, "atan": 5, "acos": 6, "atan2": 7}


def math_eval(fn, x, out, y=None, stream=None):
    """Evaluates a kernel transcendental (diagnostic, no reference counterpart)."""
    code = MATH_FN[fn] if isinstance(fn, str) else int(fn)
    n = x.numel() if hasattr(x, "numel") else int(len(x))
    check(lib.cudapic_math_eval(code, _ptr(x), _ptr(y), _ptr(out), n, _stream(stream, x)))
