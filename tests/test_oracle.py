"""CPU tests: the oracle against the reference's golden vectors and known
answers, and the self-consistency of each restated kernel."""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def test_xoshiro_golden(oracle):
    # Rust-CUDA/src/main.rs:2002-2063 test_gpu_xoshiro: 10 000 outputs from {1,1,1,1}
    gold = np.loadtxt(os.path.join(GOLDEN, "xoshiro128p_10000.txt"), dtype=np.uint64).astype(np.uint32)
    assert gold.size == 10000
    assert np.array_equal(oracle.xoshiro_stream([1, 1, 1, 1], 10000), gold)


def test_u32_to_real_bounds(oracle):
    assert oracle.u32_to_real(0) == 0.0
    assert oracle.u32_to_real(0xFFFFFFFF) == np.float32(1.0 - 2.0 ** -23)
    assert oracle.u32_to_real(0x80000000) == 0.5


def _py_next(s):
    m = 0xFFFFFFFF
    s0, s1, s2, s3 = s
    r = (s0 + s3) & m
    t = (s1 << 9) & m
    s2 ^= s0
    s3 ^= s1
    s1 ^= s2
    s0 ^= s3
    s2 ^= t
    s3 = ((s3 << 11) | (s3 >> 21)) & m
    return r, [s0, s1, s2, s3]


def test_jump_is_2_64_steps_linear_map(oracle):
    # jump() == J s with J linear over GF(2): J(a ^ b) == J a ^ J b
    a = np.array([0x12345678, 0x11112222, 0x22223333, 0x33334444], np.uint32)
    b = np.array([0x9abcdef0, 0x0badf00d, 0xdeadbeef, 0x01234567], np.uint32)
    ja, jb, jab = oracle.jump(a), oracle.jump(b), oracle.jump(a ^ b)
    assert np.array_equal(jab, ja ^ jb)


def test_seed_streams_matches_repeated_jumps(oracle):
    master = [0x12345678, 0x11112222, 0x22223333, 0x33334444]
    s = oracle.seed_streams(master, 40)
    state = np.array(master, np.uint32)
    for k in range(40):
        assert [int(p[k]) for p in s] == [int(v) for v in state]
        state = oracle.jump(state)
    with pytest.raises(ValueError):
        oracle.seed_streams([0, 0, 0, 0], 4)


def test_jump_tables_reproduce_sequential_jumps(oracle):
    """The GF(2) power tables compiled into the seeding kernel give stream
    16*m == 16*m sequential jumps (checked on the CPU)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gen_jump_tables", os.path.join(ROOT, "cudapic_b200", "csrc", "gen_jump_tables.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    tables = gen.jump_power_columns()
    master = [0x44445555, 0x55556666, 0x66667777, 0x77778888]
    ref = oracle.seed_streams(master, 16 * 37 + 1)
    v = master[0] | (master[1] << 32) | (master[2] << 64) | (master[3] << 96)
    for m in (1, 2, 5, 36, 37):
        k = 16 * m
        s = v
        for lvl, cols in enumerate(tables):
            if (k >> (lvl + gen.FIRST_LEVEL)) & 1:
                s = gen._matvec(cols, s)
        got = [(s >> (32 * w)) & 0xFFFFFFFF for w in range(4)]
        assert got == [int(p[k]) for p in ref]


@pytest.mark.parametrize("fn,lo,hi,ulps", [
    ("exp", -30.0, 5.0, 1.5), ("log", 1e-9, 1.0, 2.5), ("sin", -12.0, 12.0, 2.0), ("cos", -12.0, 12.0, 2.0),
    ("tan", -1.5, 1.5, 3.0), ("atan", -50.0, 50.0, 3.0), ("acos", -1.0, 1.0, 3.5)])
def test_math_accuracy_vs_libm(oracle, fn, lo, hi, ulps):
    rng = np.random.default_rng(7)
    x = rng.uniform(lo, hi, 200_000).astype(np.float32)
    ref = getattr(np, {"atan": "arctan", "acos": "arccos"}.get(fn, fn))(x.astype(np.float64))
    got = oracle.math_apply(fn, x).astype(np.float64)
    spacing = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    assert np.max(np.abs(got - ref) / spacing) <= ulps


def test_collision_fast_reject_bound(oracle):
    """The kernels skip exp() when u >= fl(a + 5e-7), a = nu dt: valid because
    the computed p = 1 - exp_det(-a) never exceeds a + 3.1e-7 (1 - e^-a <= a,
    exp_det within 2 ulp, 1 - y exact for y >= 1/2).  Checked densely."""
    a = np.concatenate([np.linspace(0.0, 1.0, 2_000_001), 10 ** np.linspace(-9, 0, 200_001)]).astype(np.float32)
    y = oracle.math_apply("exp", -a)
    p = (np.float32(1.0) - y).astype(np.float32)
    thr = (a + np.float32(5e-7)).astype(np.float32)
    assert np.all(p.astype(np.float64) < thr.astype(np.float64))
    # and the bound is tight enough to matter: most u >= thr for the typical a ~ 4e-3
    assert np.mean(thr[(a > 3e-3) & (a < 5e-3)]) < 6e-3


def test_atan2_quadrants(oracle):
    rng = np.random.default_rng(8)
    y = rng.uniform(-3, 3, 100_000).astype(np.float32)
    x = rng.uniform(-3, 3, 100_000).astype(np.float32)
    got = oracle.math_apply("atan2", y, x).astype(np.float64)
    ref = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    assert np.max(np.abs(got - ref)) < 5e-7


def test_phys_constants_match_reference(oracle):
    ph = oracle.phys_from_params()
    # hard-coded in the reference: NORMAL_RANGE, Rust-CUDA/src/main.rs:92
    assert ph.normal_range == np.float32(269.90040554976775)
    assert ph.inv_dx == np.float32(399 / 0.025)
    dt_e = 1.0 / 13.56e6 / 4000
    assert ph.dt_e == np.float32(dt_e)
    assert ph.factor_e == np.float32(dt_e / 9.10938356e-31 * -1.60217662e-19)


def test_hakim_convergence_order(oracle):
    # Rust-CUDA/src/main.rs:1887-1981: psi'' = 1 - 2x^2, psi(0) = psi(1) = 0,
    # exact x^2/2 - x^4/6 - x/3; second-order convergence.
    errs = []
    for n_elem in (8, 16, 32, 64):
        n = n_elem + 1
        dx = 1.0 / n_elem
        xs = np.arange(n) * dx
        src = (1.0 - 2.0 * xs * xs).astype(np.float32).astype(np.float64)
        pot = oracle.poisson_dps_flexible_f64(src, 0.0, 0.0, dx)
        exact = xs ** 2 / 2 - xs ** 4 / 6 - xs / 3
        errs.append(np.mean(np.abs(pot[1:-1] - exact[1:-1])))
    orders = [math.log(errs[i] / errs[i + 1]) / math.log(2.0) for i in range(3)]
    assert all(1.9 < o < 2.1 for o in orders), orders


def _quasi_neutral_profile(n_g, seed=3):
    ref = np.loadtxt(os.path.join(GOLDEN, "edupic_ref_density.txt"))
    xs = np.linspace(0, 1, n_g)
    ne = np.interp(xs, np.linspace(0, 1, ref.shape[0]), ref[:, 1]).astype(np.float32)
    ni = np.interp(xs, np.linspace(0, 1, ref.shape[0]), ref[:, 2]).astype(np.float32)
    return ne, ni


@pytest.mark.parametrize("n_g,tol", [(400, 1e-3), (4096, 5e-2)])
def test_scan_f32_vs_thomas(oracle, n_g, tol):
    ph = oracle.phys_from_params(n_g=n_g)
    ne, ni = _quasi_neutral_profile(n_g)
    pot_t, ef_t = oracle.poisson_thomas_f64(ne, ni, 250.0, ph)
    pot_s, ef_s = oracle.poisson_scan_f32(ne, ni, 250.0, ph)
    rel = np.linalg.norm(pot_s - pot_t) / np.linalg.norm(pot_t)
    assert rel < tol


def test_deposit_f32_vs_f64(oracle):
    ph = oracle.phys_from_params()
    rng = np.random.default_rng(11)
    x = (rng.random(200_000) * 0.025).astype(np.float32)
    d32 = oracle.get_density_f32(x, ph)
    d64 = oracle.get_density_f64(x, ph)
    assert np.linalg.norm(d32 - d64) / np.linalg.norm(d64) < 1e-5
    # total charge: every particle deposits W (interior) -> sum with doubled ends
    interior = d64[1:-1].sum() + d64[0] / 2 + d64[-1] / 2
    assert abs(interior - ph.weight_factor_d * x.size) / (ph.weight_factor_d * x.size) < 1e-12


def test_deposit_clamps_particle_at_gap_end(oracle):
    ph = oracle.phys_from_params()
    x = np.array([ph.gap, 0.0], np.float32)  # pos == N_G-1 exactly: node N_G-2 / N_G-1 cell
    d = oracle.get_density_f32(x, ph)
    assert d.shape == (400,)
    assert d[-1] > 0 and d[0] > 0


def test_move_and_compact_absorbs_only_leavers(oracle):
    ph = oracle.phys_from_params()
    from cudapic_b200.workloads import steady_state, field_profile
    x, vx, vy, vz = steady_state(100_000, 9.10938356e-31, 3.0, dt=ph.dt_e, seed=1)
    ef = field_profile(400)
    nx, nvx, nvy, nvz, src = oracle.move_and_compact(ef, x, vx, vy, vz, ph.factor_e, ph.dt_e, ph)
    assert np.all((nx >= 0) & (nx <= ph.gap))
    assert np.all(np.diff(src.astype(np.int64)) > 0)  # stable order
    assert 0 < x.size - nx.size < 300  # ~0.1 % placed to leave
    assert np.array_equal(nvy, vy[src]) and np.array_equal(nvz, vz[src])


def test_collision_decisions_vs_exact(oracle, tables):
    """The f32 decision u < 1 - exp(-nu dt) with the deterministic exp agrees
    with the exact double-precision decision except within a 1e-6 band."""
    cs, se, si = tables
    n = 200_000
    ph = oracle.phys_from_params(capacity=n + 1000)
    from cudapic_b200.workloads import steady_state
    x, vx, vy, vz = steady_state(n, 9.10938356e-31, 8.0, dt=ph.dt_e, seed=2)
    rng = [np.asarray(p) for p in oracle.seed_streams([1, 2, 3, 4], n)]
    r0 = [p.copy() for p in rng]
    cap = n + 1000
    e = [np.zeros(cap, np.float32) for _ in range(4)]
    for a, b in zip(e, (x, vx, vy, vz)):
        a[:n] = b
    ions = [np.zeros(cap, np.float32) for _ in range(4)]
    vx0, vy0, vz0 = e[1][:n].copy(), e[2][:n].copy(), e[3][:n].copy()
    events, ne, ni, dropped = oracle.check_collisions_e(se, cs, n, e, rng, ions, n, 0, ph)
    u = np.array([oracle.u32_to_real((int(a) + int(b)) & 0xFFFFFFFF) for a, b in zip(r0[0], r0[3])])
    p = np.array([oracle.p_coll_e_exact(se, a, b, c, ph) for a, b, c in zip(vx0, vy0, vz0)])
    exact = u < p
    got = events > 0
    mismatch = exact != got
    assert np.all(np.abs(u - p)[mismatch] < 1e-6)
    assert got.sum() > 100
    assert ne - n == np.sum(events == 3) and ni == np.sum(events == 3)
    assert dropped == 0


def test_wall_count_known_answers(oracle):
    """Boundary check of C/eduPIC.cc:623-667: sides by the pushed position,
    ion energies binned at floor(1/2 M v^2 / e) below 200 eV."""
    import numpy as np
    ph = oracle.phys_from_params()
    L = ph.gap
    m_half = 0.5 * 6.63352090e-26 / 1.60217662e-19
    v_of = lambda e: np.sqrt(e / m_half)  # noqa: E731
    x = np.array([-1e-6, -1e-6, L + 1e-6, L + 1e-6, 0.5 * L, 0.0, L], np.float32)
    vx = np.array([-v_of(10.5), -v_of(250.0), v_of(3.2), 0.0, 0.0, 0.0, 0.0], np.float32)
    z = np.zeros_like(x)
    counts, ip, ig = oracle.wall_count(np.zeros(400, np.float32), x, vx, z, z, 0.0, 0.0, ph, True)
    assert list(counts) == [2, 2]                       # x = 0 and x = L stay
    assert ip.sum() == 1 and ip[10] == 1                 # the 250 eV ion is counted but not binned
    assert ig.sum() == 2 and ig[3] == 1 and ig[0] == 1
    # electrons: counts only; every absorbed particle is one not kept by the push
    from cudapic_b200.workloads import field_profile, steady_state
    xs, vxs, vys, vzs = steady_state(20000, 9.10938356e-31, 5.0, dt=1.8e-11, edge_fraction=0.02, seed=3)
    ef = field_profile(400)
    c, _, _ = oracle.wall_count(ef, xs, vxs, vys, vzs, -3.2e4, 1.8e-11, ph, False)
    kept = oracle.move_and_compact(ef, xs, vxs, vys, vzs, -3.2e4, 1.8e-11, ph)[0].size
    assert int(c.sum()) == 20000 - kept and c.min() > 0


def test_algebraic_scattering_matches_angle_form(oracle, tables):
    """The fused step's scattering arithmetic (sines and cosines of the Euler
    angles, of acos(c) and of eta + pi from their algebraic forms) makes the
    same decisions, draws and spawns as the reference's angle form, and
    velocities within a few f32 ulps of the scattered speed."""
    cs, se, si = tables
    n = 100_000
    ph = oracle.phys_from_params(capacity=2 * n)
    from cudapic_b200.workloads import steady_state
    x, vx, vy, vz = steady_state(n, 9.10938356e-31, 12.0, dt=ph.dt_e, seed=5)
    # exact zeros take the special cases gx = 0 and gy = 0
    vx[:50] = 0.0
    vy[50:100] = 0.0
    vx[100:120] = 0.0
    vy[100:120] = 0.0
    out = []
    for alg in (False, True):
        rng = [np.asarray(p) for p in oracle.seed_streams([7, 8, 9, 10], 2 * n)]
        e = [np.zeros(2 * n, np.float32) for _ in range(4)]
        for a, b in zip(e, (x, vx, vy, vz)):
            a[:n] = b
        ions = [np.zeros(2 * n, np.float32) for _ in range(4)]
        r = oracle.check_collisions_e(se, cs, n, e, rng, ions, n, 0, ph, algebraic=alg)
        out.append((r, e, rng, ions))
    (ra, ea, ga, ia), (rb, eb, gb, ib) = out
    np.testing.assert_array_equal(ra[0], rb[0])
    assert ra[1:] == rb[1:]
    assert np.sum(ra[0] == 1) > 100 and np.sum(ra[0] == 3) > 10
    for p, q in zip(ga, gb):
        np.testing.assert_array_equal(p, q)
    ne = ra[1]
    np.testing.assert_array_equal(ea[0][:ne], eb[0][:ne])
    np.testing.assert_array_equal(ia[0][:ra[2]], ib[0][:ra[2]])
    for planes_a, planes_b, count in ((ea, eb, ne), (ia, ib, ra[2])):
        va = np.stack([p[:count].astype(np.float64) for p in planes_a[1:]])
        vb = np.stack([p[:count].astype(np.float64) for p in planes_b[1:]])
        speed = np.maximum(np.linalg.norm(va, axis=0), 1.0)
        assert np.max(np.abs(va - vb) / speed) < 8 * 2.0 ** -23
    scattered = np.flatnonzero(ra[0])
    assert np.count_nonzero(ea[1][scattered] != eb[1][scattered]) > 0  # the forms differ in rounding
