"""GPU parity tests: every drop-in kernel of libcudapic, called through the C
ABI on a B200, against the oracle on the same seeded inputs.

Bar per kernel (reference file:line in the kernel sources):
  RNG, seeding, EEPF, density accumulation .......... bit-exact
  move_and_compact .... survivor count and survivor set bit-exact
  check_collisions_e/i  event types, RNG states and velocities bit-exact;
                        spawned particles bit-exact as a set
  get_density ......... relative L2 <= 2e-5 vs the FP64 eduPIC deposit
  solve_poisson ....... relative L2 <= 1e-6 (FP64 sums) vs FP64 Thomas;
                        <= 1e-3 (N_G = 400) / 5e-2 (4096) in f32 mode
"""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN
from gpu_util import check_step_electrons, counter, dev, host, sorted_rows, zeros

pytestmark = pytest.mark.gpu

E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26


@pytest.fixture(scope="module")
def K(cudapic, cuda_device):
    return cudapic.kernels


@pytest.fixture(scope="module")
def dev_tables(tables, cuda_device):
    cs, se, si = tables
    return dev(cs), dev(se), dev(si)


# ---------------------------------------------------------------- RNG

def test_xoshiro_known_answer(K):
    # Rust-CUDA/src/main.rs:2002-2063 with a real assert
    gold = np.loadtxt(os.path.join(GOLDEN, "xoshiro128p_10000.txt"), dtype=np.uint64).astype(np.uint32)
    dest = zeros(5, np.uint32)
    s = [1, 1, 1, 1]
    out = np.empty(10000, np.uint32)
    for i in range(10000):
        K.xoshiro128p_test_wrapper(*s, dest)
        h = host(dest)
        out[i] = h[0]
        s = [int(v) for v in h[1:5]]
    assert np.array_equal(out, gold)


@pytest.mark.parametrize("n", [1, 17, 100_003, 4_194_304])
def test_seed_streams_bit_exact(K, oracle, n):
    master = [0x12345678, 0x11112222, 0x22223333, 0x33334444]
    planes = [zeros(n, np.uint32) for _ in range(4)]
    K.xoshiro128_seed_streams(master, n, *planes)
    ref = oracle.seed_streams(master, n)
    for p, r in zip(planes, ref):
        assert np.array_equal(host(p), r)


@pytest.mark.parametrize("fn,lo,hi", [("exp", -40.0, 5.0), ("log", 1e-9, 1.0), ("sin", -10.0, 10.0),
                                      ("cos", -10.0, 10.0), ("tan", -1.5, 1.5), ("atan", -60.0, 60.0),
                                      ("acos", -1.0, 1.0), ("atan2", -4.0, 4.0)])
def test_math_bit_exact_with_oracle(K, oracle, fn, lo, hi):
    rng = np.random.default_rng(21)
    x = rng.uniform(lo, hi, 1 << 20).astype(np.float32)
    y = rng.uniform(lo, hi, 1 << 20).astype(np.float32)
    out = zeros(x.size)
    K.math_eval(fn, dev(x), out, y=dev(y))
    ref = oracle.math_apply(fn, x, y)
    assert np.array_equal(host(out).view(np.uint32), ref.view(np.uint32))


# ---------------------------------------------------------------- deposit

@pytest.mark.parametrize("arith", ["fixed20", "f32"])
@pytest.mark.parametrize("n_g", [400, 4096])
@pytest.mark.parametrize("n", [0, 1, 1001, 100_003, 4_194_304])
def test_get_density_vs_fp64(cudapic, K, oracle, n_g, n, arith):
    flags = cudapic.FLAG_DEPOSIT_F32 if arith == "f32" else 0
    g = cudapic.grid_from_params(n_g=n_g, capacity=max(n, 4), flags=flags)
    ph = oracle.phys_from_params(n_g=n_g, capacity=max(n, 4))
    rng = np.random.default_rng(n + n_g)
    x = (rng.random(n) * 0.025).astype(np.float32)
    if n:
        x[0] = np.float32(0.025)  # exactly at the grounded electrode
    dens = zeros(n_g)
    K.get_density(dev(x) if n else zeros(4), dens, counter(n), g)
    got = host(dens).astype(np.float64)
    ref = oracle.get_density_f64(x, ph)
    if n == 0:
        assert not got.any()
        return
    # f32 restatement (same arithmetic, sequential summation order)
    r32 = oracle.get_density_f32(x, ph).astype(np.float64)
    assert np.linalg.norm(got - r32) / np.linalg.norm(r32) < 2e-5
    # FP64 eduPIC deposit: the f32 position x*inv_dx carries an absolute
    # rounding error up to N_G * 2^-24 in the CIC weights (the reference's
    # f32 arithmetic), which averages out only over many particles per node.
    tol = max(2e-5, 1.5 * n_g * 2.0 ** -24)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < tol
    # per node: absolute error bounded by the per-particle weight error
    w = ph.weight_factor_d
    assert np.max(np.abs(got - ref)) < 2.0 * w * max(1.0, np.sqrt(n / n_g)) * (n_g * 2.0 ** -24 + 1e-6) + 1e-6 * ref.max()
    if n >= 100 * n_g:   # densely populated nodes: relative error per node
        big = ref > 1e-3 * ref.max()
        assert np.max(np.abs(got[big] - ref[big]) / ref[big]) < max(1e-4, 3.0 * n_g * 2.0 ** -24)


@pytest.mark.parametrize("n_g", [400, 4096])
@pytest.mark.parametrize("n", [1, 100_003, 4_194_304])
def test_get_density_fixed_point(cudapic, K, oracle, n_g, n):
    """CUDAPIC_FLAG_DEPOSIT_FIXED_POINT: 32.32 fixed-point integer sums."""
    g = cudapic.grid_from_params(n_g=n_g, capacity=n, flags=cudapic.FLAG_DEPOSIT_FIXED_POINT)
    ph = oracle.phys_from_params(n_g=n_g, capacity=n)
    x = (np.random.default_rng(n).random(n) * 0.025).astype(np.float32)
    dens = zeros(n_g)
    K.get_density(dev(x), dens, counter(n), g)
    got = host(dens).astype(np.float64)
    r32 = oracle.get_density_f32(x, ph).astype(np.float64)
    assert np.linalg.norm(got - r32) / np.linalg.norm(r32) < 2e-5
    ref = oracle.get_density_f64(x, ph)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < max(2e-5, 1.5 * n_g * 2.0 ** -24)


def test_get_density_fixed_point_is_exact_per_cta(cudapic, K, oracle):
    """With one CTA (all of it in one cluster) the fixed-point deposit is a
    single exact integer sum: two runs give identical bits and the value is
    the exact CIC sum of the f32 fractions, rounded once."""
    saved = cudapic.get_tuning()
    try:
        cudapic.set_tuning(density_ctas_per_sm=1, density_cluster=1)
        n = 3000   # two CTAs: two f32 partial sums per node, commutative
        g = cudapic.grid_from_params(capacity=n, flags=cudapic.FLAG_DEPOSIT_FIXED_POINT)
        ph = oracle.phys_from_params(capacity=n)
        x = (np.random.default_rng(9).random(n) * 0.025).astype(np.float32)
        runs = []
        for _ in range(2):
            dens = zeros(400)
            K.get_density(dev(x), dens, counter(n), g)
            runs.append(host(dens))
        assert np.array_equal(runs[0].view(np.uint32), runs[1].view(np.uint32))
        # exact reference: sum of (1 - rem), rem with rem the f32 fraction, in exact rationals
        pos = (x * np.float32(g.inv_dx)).astype(np.float32)
        p = np.minimum(pos.astype(np.int64), 398)
        rem = (pos - p.astype(np.float32)).astype(np.float32).astype(np.float64)
        r = np.rint(rem * 2.0 ** 32)
        acc = np.zeros(400)
        np.add.at(acc, p, 2.0 ** 32 - r)
        np.add.at(acc, p + 1, r)
        exp = acc * (ph.weight_factor_d * 2.0 ** -32)
        exp[0] *= 2
        exp[-1] *= 2
        assert np.max(np.abs(runs[0] - exp) / np.maximum(exp, 1e-30)) < 1.2e-7
    finally:
        cudapic.set_tuning(**saved)


@pytest.mark.parametrize("vec", [True, False])
def test_get_density_fixed20_drains_are_exact(cudapic, K, vec):
    """Default arithmetic at its limit: one histogram copy, one CTA per SM, no
    cluster, particles in three cells with fractions up to ~1, so each copy
    is drained every round.  Equals the exact CIC sum of the 2^-20-rounded
    fractions."""
    import torch
    saved = cudapic.get_tuning()
    try:
        cudapic.set_tuning(density_copies=1, density_ctas_per_sm=1, density_cluster=1, density_threads=512)
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        n = 40 * sms * 512 * 4 + 3           # 40 rounds of float4 loads per CTA and a ragged tail
        n_g = 400
        g = cudapic.grid_from_params(n_g=n_g, capacity=n + 1)
        xs = np.array([(200 + 0.9999) * g.dx, (37 + 0.5) * g.dx, (398 + 0.9995) * g.dx], np.float32)
        x = np.resize(xs, n).astype(np.float32)
        buf = dev(np.concatenate([[0.0], x]).astype(np.float32))
        dens = zeros(n_g)
        K.get_density(buf.data_ptr() + (0 if vec else 4), dens, counter(n), g)
        if vec:
            x = np.concatenate([[0.0], x[:-1]]).astype(np.float32)
        pos = x * np.float32(g.inv_dx)
        p = np.minimum(np.floor(pos).astype(np.int64), n_g - 2)
        rem = (pos - p.astype(np.float32)).astype(np.float64)
        r = np.minimum(np.rint(rem * 2.0 ** 20), 2.0 ** 20)
        acc = np.zeros(n_g)
        np.add.at(acc, p, 2.0 ** 20 - r)
        np.add.at(acc, p + 1, r)
        exp = acc * (g.weight_factor_d * 2.0 ** -20)
        exp[0] *= 2.0
        exp[-1] *= 2.0
        got = host(dens).astype(np.float64)
        # one CTA-sum per CTA rounded to f32, then f32 atomics across CTAs
        assert np.allclose(got, exp, rtol=1e-5, atol=1e-6 * exp.max())
    finally:
        cudapic.set_tuning(**saved)


def test_get_density_unaligned_pointer(cudapic, K, oracle):
    n, n_g = 50_001, 400
    g = cudapic.grid_from_params(n_g=n_g, capacity=n + 1)
    ph = oracle.phys_from_params(n_g=n_g)
    x = (np.random.default_rng(5).random(n) * 0.025).astype(np.float32)
    buf = dev(np.concatenate([[0.0], x]).astype(np.float32))
    dens = zeros(n_g)
    K.get_density(buf.data_ptr() + 4, dens, counter(n), g)
    ref = oracle.get_density_f64(x, ph)
    assert np.linalg.norm(host(dens) - ref) / np.linalg.norm(ref) < 2e-5


def test_accumulate_density_bit_exact(cudapic, K, oracle):
    g = cudapic.grid_from_params()
    d = np.random.default_rng(3).random(400).astype(np.float32) * 1e14
    c0 = np.random.default_rng(4).random(400) * 1e16
    cum = dev(c0)
    K.accumulate_density(dev(d), cum, g)
    ref = c0.copy()
    oracle.accumulate_density(d, ref)
    assert np.array_equal(host(cum), ref)


# ---------------------------------------------------------------- Poisson

def _profile(n_g, seed):
    ref = np.loadtxt(os.path.join(GOLDEN, "edupic_ref_density.txt"))
    xs = np.linspace(0, 1, n_g)
    ne = np.interp(xs, np.linspace(0, 1, ref.shape[0]), ref[:, 1])
    ni = np.interp(xs, np.linspace(0, 1, ref.shape[0]), ref[:, 2])
    noise = np.random.default_rng(seed).normal(0, 0.02, (2, n_g))
    return (ne * (1 + noise[0])).astype(np.float32), (ni * (1 + noise[1])).astype(np.float32)


@pytest.mark.parametrize("n_g", [3, 33, 400, 1025, 4096, 16384])
@pytest.mark.parametrize("pot0", [250.0, -117.3])
def test_poisson_fp64_scan_vs_thomas(cudapic, K, oracle, n_g, pot0):
    g = cudapic.grid_from_params(n_g=n_g)
    ph = oracle.phys_from_params(n_g=n_g)
    ne, ni = _profile(n_g, n_g)
    pot, ef = zeros(n_g), zeros(n_g)
    K.solve_poisson_scan_f32(dev(ne), dev(ni), pot, ef, pot0, g)
    pt, et = oracle.poisson_thomas_f64(ne, ni, np.float32(pot0), ph)
    gp, ge = host(pot).astype(np.float64), host(ef).astype(np.float64)
    assert np.linalg.norm(gp - pt) / np.linalg.norm(pt) < 1e-6
    assert np.linalg.norm(ge - et) / np.linalg.norm(et) < 1e-5
    assert gp[0] == np.float32(pot0) and gp[-1] == 0.0


@pytest.mark.parametrize("n_g,tol", [(400, 1e-3), (4096, 5e-2)])
def test_poisson_f32_scan_vs_thomas(cudapic, K, oracle, n_g, tol):
    g = cudapic.grid_from_params(n_g=n_g, flags=cudapic.FLAG_POISSON_F32_SCAN)
    ph = oracle.phys_from_params(n_g=n_g)
    ne, ni = _profile(n_g, 1)
    pot, ef = zeros(n_g), zeros(n_g)
    K.solve_poisson_scan_f32(dev(ne), dev(ni), pot, ef, 250.0, g)
    pt, _ = oracle.poisson_thomas_f64(ne, ni, 250.0, ph)
    assert np.linalg.norm(host(pot) - pt) / np.linalg.norm(pt) < tol


def test_poisson_hakim_convergence(K, oracle):
    # Rust-CUDA/src/main.rs:1895-1981, with the assert the reference omits
    errs = []
    for n_elem in (8, 16, 32, 64):
        n = n_elem + 1
        dx = 1.0 / n_elem
        xs = np.arange(n) * dx
        src = (1.0 - 2.0 * xs * xs).astype(np.float32)
        pot = zeros(n)
        K.solve_poisson_dps_flexible(dev(src), pot, n, 0.0, 0.0, dx)
        p = host(pot).astype(np.float64)
        exact = xs ** 2 / 2 - xs ** 4 / 6 - xs / 3
        ref = oracle.poisson_dps_flexible_f64(src.astype(np.float64), 0.0, 0.0, np.float32(dx))
        assert np.max(np.abs(p - ref)) < 1e-6
        errs.append(np.mean(np.abs(p[1:-1] - exact[1:-1])))
    orders = [math.log(errs[i] / errs[i + 1]) / math.log(2.0) for i in range(3)]
    assert all(1.9 < o < 2.1 for o in orders), orders


# ---------------------------------------------------------------- push + compaction

def _population(n, species, seed, dt):
    from cudapic_b200.workloads import steady_state
    if species == "e":
        return steady_state(n, E_MASS, 3.0, dt=dt, seed=seed)
    return steady_state(n, AR_MASS, 0.03, dt=dt * 20, seed=seed)


@pytest.mark.parametrize("species", ["e", "i"])
@pytest.mark.parametrize("n", [0, 5, 2047, 2048, 2049, 100_003, 4_194_304])
@pytest.mark.parametrize("n_g", [400, 4096])
def test_move_and_compact_bit_exact(cudapic, K, oracle, species, n, n_g):
    from cudapic_b200.workloads import field_profile
    cap = max(4, (n + 3) // 4 * 4)
    g = cudapic.grid_from_params(n_g=n_g, capacity=cap)
    ph = oracle.phys_from_params(n_g=n_g, capacity=cap)
    factor, dt = (g.factor_e, g.dt_e) if species == "e" else (g.factor_i, g.dt_i)
    x, vx, vy, vz = _population(n, species, n + 7, g.dt_e)
    ef = field_profile(n_g)
    src = [dev(np.concatenate([a, np.zeros(cap - n, np.float32)])) for a in (x, vx, vy, vz)]
    dst = [zeros(cap) for _ in range(4)]
    alive = counter(0)
    K.move_and_compact(dev(ef), *src, *dst, alive, counter(n), factor, dt, g)
    m = int(host(alive)[0])
    rx, rvx, rvy, rvz, _ = oracle.move_and_compact(ef, x, vx, vy, vz, factor, dt, ph)
    assert m == rx.size
    got = [host(d)[:m] for d in dst]
    assert np.array_equal(sorted_rows(*got), sorted_rows(rx, rvx, rvy, rvz))


@pytest.mark.parametrize("n,n_g", [(5, 400), (100_003, 400), (4_194_304, 400), (1_000_001, 4096)])
def test_move_and_compact_deposit(cudapic, K, oracle, n, n_g):
    """Fused push + deposit: survivors bit-exact, and the deposited density
    equals get_density of the survivors (f32 restatement / FP64)."""
    from cudapic_b200.workloads import field_profile
    cap = (n + 3) // 4 * 4
    g = cudapic.grid_from_params(n_g=n_g, capacity=cap)
    ph = oracle.phys_from_params(n_g=n_g, capacity=cap)
    x, vx, vy, vz = _population(n, "e", n + 3, g.dt_e)
    ef = field_profile(n_g)
    src = [dev(np.concatenate([a, np.zeros(cap - n, np.float32)])) for a in (x, vx, vy, vz)]
    dst = [zeros(cap) for _ in range(4)]
    alive = counter(0)
    nd = zeros(n_g)
    K.move_and_compact_deposit(dev(ef), *src, *dst, alive, counter(n), g.factor_e, g.dt_e, nd, g)
    m = int(host(alive)[0])
    rx, rvx, rvy, rvz, _ = oracle.move_and_compact(ef, x, vx, vy, vz, g.factor_e, g.dt_e, ph)
    assert m == rx.size
    assert np.array_equal(sorted_rows(*[host(d)[:m] for d in dst]), sorted_rows(rx, rvx, rvy, rvz))
    got = host(nd).astype(np.float64)
    r32 = oracle.get_density_f32(rx, ph).astype(np.float64)
    assert np.linalg.norm(got - r32) / np.linalg.norm(r32) < 2e-5
    r64 = oracle.get_density_f64(rx, ph)
    assert np.linalg.norm(got - r64) / np.linalg.norm(r64) < max(2e-5, 1.5 * n_g * 2.0 ** -24)


def test_move_and_compact_deposit_fixed_point_copies_do_not_overflow(cudapic, K):
    """Worst case of the fixed-point fused deposit: one histogram copy, one
    CTA per SM, the particles in three cells with fractions up to ~1, and
    enough tiles per CTA that the 32-bit copies are drained many times.  The
    deposit equals the exact FP64 CIC sum (2^-21 weight quantum)."""
    saved = cudapic.get_tuning()
    try:
        cudapic.set_tuning(density_copies=1, push_ctas_per_sm=1)
        import torch
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        n = 150 * sms * 1024                 # 150 tiles per CTA: 50 drains of 3 tiles
        n_g = 400
        g = cudapic.grid_from_params(n_g=n_g, capacity=n)
        xs = np.array([(200 + 0.9999) * g.dx, (37 + 0.5) * g.dx, (398 + 0.9995) * g.dx], np.float32)
        x = np.resize(xs, n).astype(np.float32)
        z = np.zeros(n, np.float32)
        src = [dev(a) for a in (x, z, z, z)]
        dst = [zeros(n) for _ in range(4)]
        alive = counter(0)
        nd = zeros(n_g)
        K.move_and_compact_deposit(zeros(n_g), *src, *dst, alive, counter(n), g.factor_e, g.dt_e, nd, g)
        assert int(host(alive)[0]) == n
        pos = x.astype(np.float32) * np.float32(g.inv_dx)
        p = np.minimum(np.floor(pos).astype(np.int64), n_g - 2)
        rem = (pos - p.astype(np.float32)).astype(np.float64)
        exp = np.zeros(n_g)
        np.add.at(exp, p, 1.0 - rem)
        np.add.at(exp, p + 1, rem)
        exp *= g.weight_factor_d
        exp[0] *= 2.0
        exp[-1] *= 2.0
        got = host(nd).astype(np.float64)
        assert np.allclose(got, exp, rtol=1e-5, atol=0.0), np.flatnonzero(~np.isclose(got, exp, rtol=1e-5))
    finally:
        cudapic.set_tuning(**saved)


def test_check_collisions_e_deposit_spawns(cudapic, K, oracle, dev_tables, tables):
    """Spawned electrons and ions are deposited into the next-step densities."""
    cs, se, si = tables
    dcs, dse, _ = dev_tables
    n = 300_001
    cap = (2 * n + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=50, capacity=cap)
    ph = oracle.phys_from_params(n_t=50, capacity=cap)
    x, vx, vy, vz = _mcc_case(n, 60.0, 31, E_MASS)
    pad = lambda a, dt=np.float32: np.concatenate([a, np.zeros(cap - len(a), dt)])  # noqa: E731
    e_d = [dev(pad(a)) for a in (x, vx, vy, vz)]
    i_d = [zeros(cap) for _ in range(4)]
    r_d = [dev(pad(np.asarray(p), np.uint32)) for p in oracle.seed_streams([4, 4, 4, 4], n)]
    ae, ai = counter(n), counter(0)
    de, di = zeros(400), zeros(400)
    K.check_collisions_e_deposit(dse, dcs, counter(n), *e_d, *r_d, *i_d, ae, ai, de, di, g)
    ne, ni = int(host(ae)[0]), int(host(ai)[0])
    assert ne - n == ni and ni > 1000
    ex = host(e_d[0])[n:ne]
    ix = host(i_d[0])[:ni]
    for got, pos in ((host(de), ex), (host(di), ix)):
        ref = oracle.get_density_f64(pos, ph)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-5


def _wall_block():
    import ctypes as C
    import torch
    from cudapic_b200 import _lib
    return torch.zeros(C.sizeof(_lib.WallCounters) // 4, dtype=torch.int32, device="cuda")


def _wall_read(t):
    import ctypes as C
    from cudapic_b200 import _lib
    raw = host(t).view(np.uint32).tobytes()
    return _lib.WallCounters.from_buffer_copy(raw).as_dict()


@pytest.mark.parametrize("species", ["e", "i"])
@pytest.mark.parametrize("layout", ["aligned", "unaligned"])
def test_move_and_compact_wall_bit_exact(cudapic, K, oracle, species, layout):
    """Absorption counters and IFEDs fused into the push (C/eduPIC.cc:623-667)
    equal the oracle's count of the same push; called twice, they add up."""
    from cudapic_b200.workloads import field_profile, steady_state
    n = 300_001
    cap = (n + 3) // 4 * 4
    g = cudapic.grid_from_params(capacity=cap + 4)
    ph = oracle.phys_from_params(capacity=cap + 4)
    mass, temp = (E_MASS, 4.0) if species == "e" else (AR_MASS, 30.0)   # hot ions: IFED bins up to ~100 eV
    factor, dt = (g.factor_e, g.dt_e) if species == "e" else (g.factor_i, g.dt_i)
    x, vx, vy, vz = steady_state(n, mass, temp, dt=dt, edge_fraction=0.02, seed=5)
    ef = field_profile(400)
    if layout == "aligned":
        src = [dev(np.concatenate([a, np.zeros(cap + 4 - n, np.float32)])) for a in (x, vx, vy, vz)]
        ptrs = src
    else:
        src = [dev(np.concatenate([[0.0], a, np.zeros(cap + 3 - n)]).astype(np.float32)) for a in (x, vx, vy, vz)]
        ptrs = [t.data_ptr() + 4 for t in src]
    wall = _wall_block()
    for rep in range(2):
        dst = [zeros(cap + 4) for _ in range(4)]
        K.move_and_compact_wall(dev(ef), *ptrs, *dst, counter(0), counter(n), factor, dt, wall, species == "i", g)
    got = _wall_read(wall)
    counts, ip, ig = oracle.wall_count(ef, x, vx, vy, vz, factor, dt, ph, species == "i")
    assert counts.min() > 1000
    assert (got["abs_pow"], got["abs_gnd"]) == (2 * int(counts[0]), 2 * int(counts[1]))
    if species == "i":
        assert ip.sum() > 1000 and ig.sum() > 1000
        assert np.array_equal(got["ifed_pow"], 2 * ip) and np.array_equal(got["ifed_gnd"], 2 * ig)
    else:
        assert not got["ifed_pow"].any() and not got["ifed_gnd"].any()


def test_move_and_compact_unaligned_uses_reference_layout(cudapic, K, oracle):
    from cudapic_b200.workloads import field_profile
    n, n_g = 70_001, 400
    g = cudapic.grid_from_params(n_g=n_g, capacity=n + 1)
    ph = oracle.phys_from_params(n_g=n_g)
    x, vx, vy, vz = _population(n, "e", 9, g.dt_e)
    ef = field_profile(n_g)
    srcb = [dev(np.concatenate([[0.0], a]).astype(np.float32)) for a in (x, vx, vy, vz)]
    dst = [zeros(n + 1) for _ in range(4)]
    alive = counter(0)
    K.move_and_compact(dev(ef), *[b.data_ptr() + 4 for b in srcb], *dst, alive, counter(n), g.factor_e, g.dt_e, g)
    m = int(host(alive)[0])
    ref = oracle.move_and_compact(ef, x, vx, vy, vz, g.factor_e, g.dt_e, ph)
    assert m == ref[0].size
    assert np.array_equal(sorted_rows(*[host(d)[:m] for d in dst]), sorted_rows(*ref[:4]))


def test_move_and_compact_appends_to_counter(cudapic, K, oracle):
    """alive_counter is an append cursor: survivors land after its start value."""
    from cudapic_b200.workloads import field_profile
    n = 10_000
    g = cudapic.grid_from_params(capacity=2 * n)
    x, vx, vy, vz = _population(n, "e", 3, g.dt_e)
    src = [dev(np.concatenate([a, np.zeros(n, np.float32)])) for a in (x, vx, vy, vz)]
    dst = [dev(np.full(2 * n, -1.0, np.float32)) for _ in range(4)]
    alive = counter(123)
    K.move_and_compact(dev(field_profile(400)), *src, *dst, alive, counter(n), g.factor_e, g.dt_e, g)
    m = int(host(alive)[0]) - 123
    hx = host(dst[0])
    assert np.all(hx[:123] == -1.0) and np.all(hx[123:123 + m] >= 0) and np.all(hx[123 + m:] == -1.0)


# ---------------------------------------------------------------- collisions

def _mcc_case(n, temp_ev, seed, mass):
    from cudapic_b200.workloads import steady_state
    return steady_state(n, mass, temp_ev, seed=seed, edge_fraction=0.0)


class _Shifted:
    """A device buffer viewed from element 1 on: a pointer that is not
    16-byte aligned, which routes the kernels to their non-bulk-copy path."""

    def __init__(self, t):
        self.t = t

    def data_ptr(self):
        return self.t.data_ptr() + 4

    def host(self):
        return host(self.t)[1:]


def _dev_layout(a, layout):
    if layout == "aligned":
        return dev(a)
    return _Shifted(dev(np.concatenate([np.zeros(1, a.dtype), a])))


def _read(d):
    return d.host() if isinstance(d, _Shifted) else host(d)


@pytest.mark.parametrize("layout", ["aligned", "unaligned"])
@pytest.mark.parametrize("n,n_t,temp", [(1, 4000, 30.0), (4099, 200, 30.0), (300_001, 4000, 20.0),
                                        (300_001, 100, 60.0), (300_001, 20, 80.0), (4_194_304, 4000, 3.0)])
def test_check_collisions_e_bit_exact(cudapic, K, oracle, dev_tables, tables, n, n_t, temp, layout):
    cs, se, si = tables
    dcs, dse, _ = dev_tables
    n_i0 = 1000
    cap = (n + n // 2 + 1024 + 3) // 4 * 4   # a multiple of 4: the bulk-copy path when aligned
    g = cudapic.grid_from_params(n_t=n_t, capacity=cap)
    ph = oracle.phys_from_params(n_t=n_t, capacity=cap)
    x, vx, vy, vz = _mcc_case(n, temp, n, E_MASS)
    rng = [np.asarray(p) for p in oracle.seed_streams([9, 8, 7, 6], n)]
    pad = lambda a, dt=np.float32: np.concatenate([a, np.zeros(cap - len(a), dt)])
    e_h = [pad(a) for a in (x, vx, vy, vz)]
    i_h = [pad(np.full(n_i0, 0.0125, np.float32)) for _ in range(4)]
    r_h = [pad(p, np.uint32) for p in rng]
    e_d = [_dev_layout(a, layout) for a in e_h]
    i_d = [_dev_layout(a, layout) for a in i_h]
    r_d = [_dev_layout(a, layout) for a in r_h]
    alive_e, alive_i = counter(n), counter(n_i0)
    events = zeros(max(n, 1), np.uint8)
    K.check_collisions_e(dse, dcs, counter(n), *e_d, *r_d, *i_d, alive_e, alive_i, g, events=events)
    ev_ref, ne_ref, ni_ref, dropped = oracle.check_collisions_e(se, cs, n, e_h, r_h, i_h, n, n_i0, ph)
    assert dropped == 0
    ge = host(events)[:n]
    assert np.array_equal(ge, ev_ref)
    if n > 4000:
        assert (ge > 0).sum() > 10
    ne, ni = int(host(alive_e)[0]), int(host(alive_i)[0])
    assert ne == ne_ref and ni == ni_ref
    for d, h in zip(r_d, r_h):
        assert np.array_equal(_read(d)[:n], h[:n])
    ge_arr = [_read(d) for d in e_d]
    for a, h in zip(ge_arr, e_h):
        assert np.array_equal(a[:n].view(np.uint32), h[:n].view(np.uint32))
    # spawned electrons and ions: same set, order unspecified
    assert np.array_equal(sorted_rows(*[a[n:ne] for a in ge_arr]), sorted_rows(*[h[n:ne] for h in e_h]))
    gi_arr = [_read(d) for d in i_d]
    assert np.array_equal(sorted_rows(*[a[n_i0:ni] for a in gi_arr]), sorted_rows(*[h[n_i0:ni] for h in i_h]))


@pytest.mark.parametrize("n,n_t,temp", [(1, 4000, 30.0), (4099, 200, 30.0), (300_001, 100, 60.0),
                                        (1_000_003, 20, 80.0), (4_194_304, 4000, 3.0)])
def test_step_electrons_bit_exact(cudapic, K, oracle, dev_tables, tables, n, n_t, temp):
    """Fused electron step against the oracle's move_and_compact followed by
    its check_collisions_e over the survivors, each survivor drawing from the
    RNG stream of its source slot (gpu_util.check_step_electrons)."""
    from cudapic_b200.workloads import field_profile, steady_state
    cap = (2 * n + 4096 + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=n_t, capacity=cap)
    ph = oracle.phys_from_params(n_t=n_t, capacity=cap)
    x, vx, vy, vz = steady_state(n, E_MASS, temp, dt=g.dt_e, seed=n + 11)
    m, ne, ni = check_step_electrons(K, oracle, tables, dev_tables, g, ph, x, vx, vy, vz, field_profile(400), cap)
    if n > 100_000 and n_t <= 100:
        assert m < n and ne > m and ni > 1000   # absorption and ionization both exercised


@pytest.mark.parametrize("n,n_t,temp,dead", [(1, 4000, 3.0, 0.0), (4093, 4000, 3.0, 0.05), (300_001, 100, 30.0, 0.0),
                                             (300_001, 100, 30.0, 0.02), (300_001, 40, 30.0, 0.0),
                                             (1_000_003, 4000, 3.0, 0.01), (4_194_304, 4000, 3.0, 0.0)])
def test_step_electrons_inplace_bit_exact(cudapic, K, oracle, dev_tables, tables, n, n_t, temp, dead):
    """In-place electron step (stream + scatter pass) against the oracle's
    move_and_compact + check_collisions_e over the live slots, every electron
    keeping its slot (gpu_util.check_step_inplace); slots emptied by earlier
    in-place steps are skipped."""
    from cudapic_b200.workloads import field_profile, steady_state
    from gpu_util import check_step_inplace, dead_mask
    cap = (2 * n + 4096 + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=n_t, capacity=cap)
    ph = oracle.phys_from_params(n_t=n_t, capacity=cap)
    x, vx, vy, vz = steady_state(n, E_MASS, temp, dt=g.dt_e, seed=n + 13)
    m, ne, ni, nc = check_step_inplace(K, oracle, tables, dev_tables, g, ph, x, vx, vy, vz, field_profile(400), cap,
                                       dead_mask(n, dead))
    if n > 100_000 and n_t <= 100:
        assert m < n and ne > n and ni > 1000 and nc > 1000   # absorption, collisions and ionization exercised


@pytest.mark.parametrize("n_g", [2048, 4096, 16384])
def test_step_electrons_inplace_large_grid(cudapic, K, oracle, dev_tables, tables, n_g):
    """Large grids: the in-place step deposits into one f32 histogram per
    CTA (no fixed-point copies); slots, RNG states and spawns stay bit-exact,
    the density within the f32 deposit tolerance max(2e-5, 1.5 N_G 2^-24)."""
    from cudapic_b200.workloads import field_profile, steady_state
    from gpu_util import check_step_inplace, dead_mask
    n = 600_001
    cap = (2 * n + 4096 + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=200, n_g=n_g, capacity=cap)
    ph = oracle.phys_from_params(n_t=200, n_g=n_g, capacity=cap)
    x, vx, vy, vz = steady_state(n, E_MASS, 20.0, dt=g.dt_e, seed=n_g + 3)
    check_step_inplace(K, oracle, tables, dev_tables, g, ph, x, vx, vy, vz, field_profile(n_g), cap,
                       dead_mask(n, 0.01), dens_tol=max(2e-5, 1.5 * n_g * 2.0 ** -24))


@pytest.mark.parametrize("n,dead", [(4093, 0.05), (300_001, 0.02)])
def test_step_electrons_skips_emptied_slots(cudapic, K, oracle, dev_tables, tables, n, dead):
    """The compacting fused step drops the slots an in-place step emptied."""
    from cudapic_b200.workloads import field_profile, steady_state
    from gpu_util import check_step_electrons_with_dead, dead_mask
    cap = (2 * n + 4096 + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=100, capacity=cap)
    ph = oracle.phys_from_params(n_t=100, capacity=cap)
    x, vx, vy, vz = steady_state(n, E_MASS, 30.0, dt=g.dt_e, seed=n + 17)
    check_step_electrons_with_dead(K, oracle, tables, dev_tables, g, ph, x, vx, vy, vz, field_profile(400), cap,
                                   dead_mask(n, dead))


def test_step_electrons_rejects_unaligned_planes(cudapic, K, dev_tables, tables):
    _, se, _ = tables
    dcs, dse, _ = dev_tables
    g = cudapic.grid_from_params(capacity=1024)
    b = [zeros(1025) for _ in range(8)]
    r = [zeros(1025, np.uint32) for _ in range(4)]
    with pytest.raises(cudapic.CudapicError):
        K.step_electrons(zeros(400), *[t.data_ptr() + 4 for t in b[:4]], *b[4:], *r, dse, dcs, float(se.max()),
                         *[zeros(1024) for _ in range(4)], counter(0), counter(10), counter(0), zeros(400),
                         zeros(400), g)


@pytest.mark.parametrize("bounded", [False, True])
@pytest.mark.parametrize("layout", ["aligned", "unaligned"])
@pytest.mark.parametrize("n,n_t,temp", [(1, 4000, 1.0), (65_537, 4000, 0.03), (300_001, 200, 2.0),
                                        (300_001, 20, 20.0), (4_194_304, 4000, 0.03)])
def test_check_collisions_i_bit_exact(cudapic, K, oracle, dev_tables, tables, n, n_t, temp, layout, bounded):
    """bounded: the entry given max(sigma_tot_i), whose ions skip the
    target's transcendentals below the certain-rejection bound -- the same
    events, RNG states and velocities."""
    cs, se, si = tables
    dcs, _, dsi = dev_tables
    cap = (n + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=n_t, capacity=cap)
    ph = oracle.phys_from_params(n_t=n_t, capacity=cap)
    _, vx, vy, vz = _mcc_case(n, temp, n + 1, AR_MASS)
    rng = [np.asarray(p) for p in oracle.seed_streams([5, 6, 7, 8], n)]
    pad = lambda a, dt=np.float32: np.concatenate([a, np.zeros(cap - len(a), dt)])
    v_h = [pad(a) for a in (vx, vy, vz)]
    r_h = [pad(p, np.uint32) for p in rng]
    v_d = [_dev_layout(a, layout) for a in v_h]
    r_d = [_dev_layout(a, layout) for a in r_h]
    events = zeros(n, np.uint8)
    K.check_collisions_i(dsi, dcs, counter(n), *v_d, *r_d, g, events=events,
                         sigma_max_i=float(si.max()) if bounded else None)
    ev_ref = oracle.check_collisions_i(si, cs, n, v_h, r_h, ph)
    assert np.array_equal(host(events), ev_ref)
    if n > 60_000:
        assert (ev_ref > 0).sum() > 10
    for d, h in zip(r_d, r_h):
        assert np.array_equal(_read(d)[:n], h[:n])
    for d, h in zip(v_d, v_h):
        assert np.array_equal(_read(d)[:n].view(np.uint32), h[:n].view(np.uint32))


def test_spawn_capacity_is_enforced(cudapic, K, oracle, dev_tables, tables):
    """Ionization spawns beyond capacity are dropped and flagged, never
    written past the buffers (the reference writes unbounded)."""
    cs, se, si = tables
    dcs, dse, _ = dev_tables
    n, cap, guard = 200_000, 200_032, 4096
    flag = zeros(1, np.uint32)
    g = cudapic.grid_from_params(n_t=50, capacity=cap)
    g.dev_err = flag.data_ptr()
    x, vx, vy, vz = _mcc_case(n, 60.0, 17, E_MASS)
    pad = lambda a, dt=np.float32: np.concatenate([a, np.full(cap + guard - len(a), 7.0, dt)])
    e_d = [dev(pad(a)) for a in (x, vx, vy, vz)]
    i_d = [dev(pad(np.zeros(cap - 16, np.float32))) for _ in range(4)]
    r_d = [dev(np.concatenate([p, np.zeros(guard, np.uint32)])) for p in oracle.seed_streams([1, 3, 5, 7], cap)]
    alive_e, alive_i = counter(n), counter(cap - 16)
    K.check_collisions_e(dse, dcs, counter(n), *e_d, *r_d, *i_d, alive_e, alive_i, g)
    assert int(host(alive_e)[0]) <= cap and int(host(alive_i)[0]) <= cap
    bits = int(host(flag)[0])
    assert bits & cudapic.DEVERR_SPAWN_E and bits & cudapic.DEVERR_SPAWN_I
    for d in e_d + i_d:
        assert np.all(host(d)[cap:] == 7.0)


# ---------------------------------------------------------------- diagnostics

def test_accumulate_eepf_bit_exact(cudapic, K, oracle):
    from cudapic_b200.workloads import field_profile
    n = 500_000
    g = cudapic.grid_from_params(capacity=n)
    ph = oracle.phys_from_params(capacity=n)
    x, vx, vy, vz = _population(n, "e", 4, g.dt_e)
    ef = field_profile(400)
    eepf = zeros(2000, np.uint32)
    K.accumulate_eepf(dev(x), dev(vx), dev(vy), dev(vz), dev(ef), counter(n), eepf, g)
    ref = np.zeros(2000, np.uint32)
    oracle.accumulate_eepf(x, vx, vy, vz, ef, n, ref, ph)
    assert ref.sum() > 10_000
    assert np.array_equal(host(eepf), ref)
