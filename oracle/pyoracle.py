"""ctypes bindings of ``libcudapic_oracle.so`` (test infrastructure only).

Each wrapper takes and returns numpy arrays and mirrors one function of
``cudapic_oracle.h``; see that header for the reference file:line each one
restates.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcudapic_oracle.so")
REF_DIR = os.path.join(_HERE, "_ref")
CS_RANGES = 1_000_000
N_EEPF = 2000
N_IFED = 200

__all__ = [
    "lib", "build", "OrcParams", "OrcPhys", "default_params", "phys_from_params", "wall_count", "N_IFED",
    "xoshiro_stream", "u32_to_real", "jump", "seed_streams", "math_apply",
    "cross_sections", "get_density_f32", "get_density_f64", "poisson_thomas_f64",
    "poisson_scan_f32", "poisson_dps_flexible_f64", "move_and_compact",
    "check_collisions_e", "check_collisions_i", "p_coll_e_exact",
    "accumulate_density", "accumulate_eepf", "xt_accumulate", "xt_normalise", "REF_DIR", "CS_RANGES", "N_EEPF",
    "MATH_FN", "SensState", "sens_run", "sens_poisson_adjoint",
]

MATH_FN = {"exp": 0, "log": 1, "sin": 2, "cos": 3, "tan": 4, "atan": 5, "acos": 6, "atan2": 7}


class OrcParams(C.Structure):
    _fields_ = [
        ("n_g", C.c_uint32), ("n_t", C.c_uint32), ("n_sub", C.c_uint32), ("capacity", C.c_uint32),
        ("frequency", C.c_double), ("voltage", C.c_double), ("gap", C.c_double),
        ("pressure", C.c_double), ("temperature", C.c_double), ("weight", C.c_double),
        ("electrode_area", C.c_double),
    ]


class OrcPhys(C.Structure):
    _fields_ = [
        ("n_g", C.c_uint32), ("capacity", C.c_uint32),
        ("inv_dx", C.c_float), ("weight_factor", C.c_float), ("gap", C.c_float),
        ("dt_e", C.c_float), ("dt_i", C.c_float), ("factor_e", C.c_float), ("factor_i", C.c_float),
        ("e_charge", C.c_float), ("alpha", C.c_float), ("half_dx_over_eps", C.c_float),
        ("half_inv_dx", C.c_float), ("normal_range", C.c_float), ("f1", C.c_float), ("f2", C.c_float),
        ("half_me_over_e", C.c_float), ("half_mu_over_e", C.c_float), ("min_x", C.c_float),
        ("max_x", C.c_float), ("eepf_half_kick", C.c_float),
        ("dx", C.c_double), ("weight_factor_d", C.c_double), ("gas_density", C.c_double),
        ("dt_e_d", C.c_double), ("dt_i_d", C.c_double), ("voltage", C.c_double), ("omega", C.c_double),
        ("n_t", C.c_uint32), ("n_sub", C.c_uint32),
    ]


class OrcSensIo(C.Structure):
    _fields_ = [
        ("x", C.c_void_p * 2), ("vx", C.c_void_p * 2), ("vy", C.c_void_p * 2), ("vz", C.c_void_p * 2),
        ("rng", (C.c_void_p * 4) * 2), ("n", C.c_uint32 * 2), ("capacity", C.c_uint32),
        ("dev_err", C.c_uint32),
    ]


def build():
    """Compile the oracle library with its Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE, "libcudapic_oracle.so"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def _declare(L):
    P = C.POINTER
    L.orc_params_default.argtypes = [P(OrcParams)]
    L.orc_phys_from_params.argtypes = [P(OrcParams), P(OrcPhys)]
    L.orc_xoshiro128p_next.argtypes = [_u32p]
    L.orc_xoshiro128p_next.restype = C.c_uint32
    L.orc_xoshiro128p_stream.argtypes = [_u32p, C.c_uint32, _u32p]
    L.orc_u32_to_real.argtypes = [C.c_uint32]
    L.orc_u32_to_real.restype = C.c_float
    L.orc_jump.argtypes = [_u32p]
    L.orc_seed_streams.argtypes = [_u32p, C.c_uint32, _u32p, _u32p, _u32p, _u32p]
    L.orc_seed_streams.restype = C.c_int
    L.orc_math_apply.argtypes = [C.c_int, _f32p, _f32p, _f32p, C.c_uint32]
    L.orc_cross_sections.argtypes = [C.c_double, _f32p, _f32p, _f32p]
    L.orc_get_density_f32.argtypes = [_f32p, C.c_uint32, _f32p, P(OrcPhys)]
    L.orc_get_density_f64.argtypes = [_f32p, C.c_uint32, _f64p, P(OrcPhys)]
    L.orc_poisson_thomas_f64.argtypes = [_f32p, _f32p, C.c_double, _f64p, _f64p, P(OrcPhys)]
    L.orc_poisson_scan_f32.argtypes = [_f32p, _f32p, C.c_float, _f32p, _f32p, P(OrcPhys)]
    L.orc_poisson_dps_flexible_f64.argtypes = [_f64p, _f64p, C.c_uint32, C.c_double, C.c_double, C.c_double]
    L.orc_move_and_compact.argtypes = [_f32p] + [_f32p] * 8 + [C.c_uint32, C.c_float, C.c_float,
                                                              P(OrcPhys), _u32p]
    L.orc_move_and_compact.restype = C.c_uint32
    L.orc_wall_count.argtypes = [_f32p] * 5 + [C.c_uint32, C.c_float, C.c_float, P(OrcPhys), C.c_int,
                                               _u64p, _u32p, _u32p]
    L.orc_wall_count.restype = None
    L.orc_check_collisions_e.argtypes = ([_f32p, _f32p, C.c_uint32] + [_f32p] * 4 + [_u32p] * 4 +
                                         [_f32p] * 4 + [P(C.c_uint32), P(C.c_uint32), P(OrcPhys),
                                                        _u8p, P(C.c_uint32)])
    L.orc_check_collisions_e_alg.argtypes = L.orc_check_collisions_e.argtypes
    L.orc_check_collisions_i.argtypes = ([_f32p, _f32p, C.c_uint32] + [_f32p] * 3 + [_u32p] * 4 +
                                         [P(OrcPhys), _u8p])
    L.orc_p_coll_e_exact.argtypes = [_f32p, C.c_float, C.c_float, C.c_float, P(OrcPhys)]
    L.orc_p_coll_e_exact.restype = C.c_double
    L.orc_accumulate_density.argtypes = [_f32p, _f64p, C.c_uint32]
    L.orc_accumulate_eepf.argtypes = [_f32p] * 5 + [C.c_uint32, _u32p, P(OrcPhys)]
    L.orc_xt_accumulate.argtypes = [_f32p] * 5 + [C.c_uint32, C.c_int, _f32p, P(OrcPhys), _f64p]
    L.orc_sens_poisson_adjoint.argtypes = [_f64p, P(OrcPhys), _f64p, _f64p]
    L.orc_sens_poisson_adjoint.restype = C.c_double
    L.orc_sens_run.argtypes = [P(OrcPhys), _f32p, _f32p, _f32p, C.c_double, C.c_uint32, C.c_uint32, C.c_int,
                               P(OrcSensIo),
                               C.POINTER(C.c_double), C.POINTER(C.c_double)]


def default_params(**overrides):
    p = OrcParams()
    lib().orc_params_default(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def phys_from_params(p=None, **overrides):
    if p is None:
        p = default_params(**overrides)
    ph = OrcPhys()
    lib().orc_phys_from_params(C.byref(p), C.byref(ph))
    return ph


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def xoshiro_stream(seed, n):
    out = np.empty(n, np.uint32)
    lib().orc_xoshiro128p_stream(_u32(seed), n, out)
    return out


def u32_to_real(x):
    return lib().orc_u32_to_real(int(x))


def jump(state):
    s = _u32(state).copy()
    lib().orc_jump(s)
    return s


def seed_streams(master, n):
    planes = [np.empty(n, np.uint32) for _ in range(4)]
    rc = lib().orc_seed_streams(_u32(master), n, *planes)
    if rc != 0:
        raise ValueError("xoshiro128+ master state must not be all zero")
    return planes


def math_apply(fn, x, y=None):
    x = _f32(x)
    y = _f32(y if y is not None else np.zeros_like(x))
    out = np.empty_like(x)
    lib().orc_math_apply(MATH_FN[fn] if isinstance(fn, str) else fn, x, y, out, x.size)
    return out


def cross_sections(gas_density):
    cs = np.empty(5 * CS_RANGES, np.float32)
    se = np.empty(CS_RANGES, np.float32)
    si = np.empty(CS_RANGES, np.float32)
    lib().orc_cross_sections(float(gas_density), cs, se, si)
    return cs, se, si


def get_density_f32(x, ph):
    x = _f32(x)
    d = np.empty(ph.n_g, np.float32)
    lib().orc_get_density_f32(x, x.size, d, C.byref(ph))
    return d


def get_density_f64(x, ph):
    x = _f32(x)
    d = np.empty(ph.n_g, np.float64)
    lib().orc_get_density_f64(x, x.size, d, C.byref(ph))
    return d


def poisson_thomas_f64(e_density, i_density, pot0, ph):
    pot = np.empty(ph.n_g, np.float64)
    ef = np.empty(ph.n_g, np.float64)
    lib().orc_poisson_thomas_f64(_f32(e_density), _f32(i_density), float(pot0), pot, ef, C.byref(ph))
    return pot, ef


def poisson_scan_f32(e_density, i_density, pot0, ph):
    pot = np.empty(ph.n_g, np.float32)
    ef = np.empty(ph.n_g, np.float32)
    lib().orc_poisson_scan_f32(_f32(e_density), _f32(i_density), float(pot0), pot, ef, C.byref(ph))
    return pot, ef


def poisson_dps_flexible_f64(source, psi_left, psi_right, dx):
    source = np.ascontiguousarray(source, np.float64)
    pot = np.empty_like(source)
    lib().orc_poisson_dps_flexible_f64(source, pot, source.size, psi_left, psi_right, dx)
    return pot


def move_and_compact(efield, x, vx, vy, vz, factor, dt, ph):
    """Returns (x, vx, vy, vz, src_index) of the survivors in index order."""
    n = len(x)
    out = [np.empty(max(n, 1), np.float32) for _ in range(4)]
    idx = np.empty(max(n, 1), np.uint32)
    m = lib().orc_move_and_compact(_f32(efield), _f32(x), _f32(vx), _f32(vy), _f32(vz), *out,
                                   n, float(factor), float(dt), C.byref(ph), idx)
    return tuple(a[:m] for a in out) + (idx[:m],)


def wall_count(efield, x, vx, vy, vz, factor, dt, ph, ions):
    """Absorption counts (powered, grounded) and IFEDs of one push
    (C/eduPIC.cc:623-667)."""
    counts = np.zeros(2, np.uint64)
    ifed_pow = np.zeros(N_IFED, np.uint32)
    ifed_gnd = np.zeros(N_IFED, np.uint32)
    lib().orc_wall_count(_f32(efield), _f32(x), _f32(vx), _f32(vy), _f32(vz), len(x), float(factor), float(dt),
                         C.byref(ph), 1 if ions else 0, counts, ifed_pow, ifed_gnd)
    return counts, ifed_pow, ifed_gnd


def check_collisions_e(sigma_tot_e, cs, n_active, e, rng, ions, n_e, n_i, ph, algebraic=False):
    """In-place MCC of electrons.  e = [x, vx, vy, vz] (capacity-sized float32
    arrays), rng = 4 uint32 planes, ions = [x, vx, vy, vz] of the ions.
    algebraic: the fused step's scattering arithmetic.  Returns (events,
    n_e, n_i, dropped)."""
    ne = C.c_uint32(n_e)
    ni = C.c_uint32(n_i)
    dropped = C.c_uint32(0)
    events = np.zeros(max(n_active, 1), np.uint8)
    fn = lib().orc_check_collisions_e_alg if algebraic else lib().orc_check_collisions_e
    fn(sigma_tot_e, cs, n_active, *e, *rng, *ions, C.byref(ne), C.byref(ni), C.byref(ph), events, C.byref(dropped))
    return events[:n_active], ne.value, ni.value, dropped.value


def check_collisions_i(sigma_tot_i, cs, n_active, v, rng, ph):
    events = np.zeros(max(n_active, 1), np.uint8)
    lib().orc_check_collisions_i(sigma_tot_i, cs, n_active, *v, *rng, C.byref(ph), events)
    return events[:n_active]


def p_coll_e_exact(sigma_tot_e, vx, vy, vz, ph):
    return lib().orc_p_coll_e_exact(sigma_tot_e, float(vx), float(vy), float(vz), C.byref(ph))


def accumulate_density(density, cumul):
    lib().orc_accumulate_density(_f32(density), cumul, cumul.size)


def accumulate_eepf(x, vx, vy, vz, efield, n_active, eepf, ph):
    lib().orc_accumulate_eepf(_f32(x), _f32(vx), _f32(vy), _f32(vz), _f32(efield), n_active, eepf,
                              C.byref(ph))


def xt_accumulate(efield, x, vx, vy, vz, ions, cs_ion, ph):
    """One step of eduPIC's XT measurement branch for one species: an array
    [3 or 4, n_g] of the weight, velocity, energy (and ionization-rate) sums."""
    n_g = ph.n_g
    out = np.zeros(4 * n_g, np.float64)  # the ions leave the rate row untouched
    cs = _f32(cs_ion if cs_ion is not None else np.zeros(1, np.float32))
    lib().orc_xt_accumulate(_f32(efield), _f32(x), _f32(vx), _f32(vy), _f32(vz), len(x), 1 if ions else 0, cs,
                            C.byref(ph), out)
    return out.reshape(4, n_g)[:3 if ions else 4]


def xt_normalise(raw, n_t, n_xt, measure_steps, gap, n_g, frequency, weight, electrode_area):
    """norm_all_xt, C/eduPIC.cc:864-903: the eleven quantities (pot, efield,
    ne, ni, je, ji, powere, poweri, meanee, meanei, ioniz) from the raw sums
    raw[name] ([n_g, n_xt] each: count_e, ue, meanee, ioniz, count_i, ui,
    meanei, pot, efield, ne, ni)."""
    e_charge = 1.60217662e-19
    cycles = measure_steps / n_t
    dx = gap / (n_g - 1)
    f1 = n_xt / (cycles * n_t)
    f2 = weight / (electrode_area * dx) / (cycles * ((1.0 / frequency) / n_xt))
    out = {k: raw[k] * f1 for k in ("pot", "efield", "ne", "ni")}
    ce, ci = raw["count_e"], raw["count_i"]
    with np.errstate(invalid="ignore", divide="ignore"):
        ue = np.where(ce > 0, raw["ue"] / ce, 0.0)
        ui = np.where(ci > 0, raw["ui"] / ci, 0.0)
        out["je"] = np.where(ce > 0, -ue * out["ne"] * e_charge, 0.0)
        out["meanee"] = np.where(ce > 0, raw["meanee"] / ce, 0.0)
        out["ioniz"] = np.where(ce > 0, raw["ioniz"] * f2, 0.0)
        out["ji"] = np.where(ci > 0, ui * out["ni"] * e_charge, 0.0)
        out["meanei"] = np.where(ci > 0, raw["meanei"] / ci, 0.0)
    out["powere"] = out["je"] * out["efield"]
    out["poweri"] = out["ji"] * out["efield"]
    return out


class SensState:
    """Both species in their slots for the sensitivity model: planes
    [x, vx, vy, vz] (float32, capacity), RNG planes (4 uint32 per species),
    slot counts n = [n_e, n_i]."""

    def __init__(self, capacity, electrons, ions, rng_e, rng_i):
        self.capacity = capacity
        self.p = []
        for parts in (electrons, ions):
            planes = [np.zeros(capacity, np.float32) for _ in range(4)]
            for a, b in zip(planes, parts):
                a[:len(b)] = b
            self.p.append(planes)
        self.rng = [[np.ascontiguousarray(np.asarray(r, np.uint32)[:capacity]).copy() for r in rr]
                    for rr in (rng_e, rng_i)]
        self.n = [len(electrons[0]), len(ions[0])]
        self.dev_err = 0

    def copy(self):
        c = SensState.__new__(SensState)
        c.capacity = self.capacity
        c.p = [[a.copy() for a in planes] for planes in self.p]
        c.rng = [[r.copy() for r in rr] for rr in self.rng]
        c.n = list(self.n)
        c.dev_err = self.dev_err
        return c


def sens_run(ph, tables, voltage, steps, state, f64=False, grad=True, horizon=0):
    """Runs the slot-form model in place on `state` (a SensState); returns
    (obs, grad): obs = [J_P W/m^3, J_G 1/(m^2 s)], grad = d obs / d voltage
    by the pathwise adjoint (None without grad), restarted every `horizon`
    steps (0: over the whole window)."""
    cs, sig_e, sig_i = tables
    io = OrcSensIo()
    for k in range(2):
        io.x[k], io.vx[k], io.vy[k], io.vz[k] = [a.ctypes.data for a in state.p[k]]
        for c in range(4):
            io.rng[k][c] = state.rng[k][c].ctypes.data
        io.n[k] = state.n[k]
    io.capacity = state.capacity
    obs = (C.c_double * 2)()
    g = (C.c_double * 2)()
    rc = lib().orc_sens_run(C.byref(ph), _f32(sig_e), _f32(sig_i), _f32(cs), float(voltage), int(steps),
                            int(horizon), 1 if f64 else 0, C.byref(io), obs, g if grad else None)
    if rc != 0:
        raise ValueError("orc_sens_run: bad arguments")
    state.n = [io.n[0], io.n[1]]
    state.dev_err = io.dev_err
    return list(obs), (list(g) if grad else None)


def sens_poisson_adjoint(eb, ph):
    """(neb, nib, pot0b): adjoints of the electron and ion densities and of
    pot0 for the field adjoint eb (the oracle's Poisson adjoint)."""
    eb = np.ascontiguousarray(eb, np.float64)
    neb = np.zeros(ph.n_g, np.float64)
    nib = np.zeros(ph.n_g, np.float64)
    p0 = lib().orc_sens_poisson_adjoint(eb, C.byref(ph), neb, nib)
    return neb, nib, p0
