"""GPU tests of the batched path: discharges stepped in lockstep by one
launch per kernel (cudapic_batch_*) against the same discharges stepped
alone by the fused driver."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26

# (n_g, electrons, ions, voltage, pressure, gap): ragged counts (not multiples
# of 4, one discharge without electrons, one with a single one), mixed grids.
# Capacities stay <= 2048, so that the priming deposit runs in one CTA
# cluster and both paths start from bit-identical densities.
CASES = [
    (400, 1500, 1400, 250.0, 10.0, 0.025),
    (200, 997, 1003, 120.0, 30.0, 0.018),
    (800, 0, 900, 480.0, 6.0, 0.038),
    (400, 1, 5, 300.0, 12.0, 0.022),
    (800, 1789, 1600, 200.0, 45.0, 0.031),
    (200, 1023, 1021, 400.0, 8.0, 0.016),
    (400, 642, 700, 350.0, 20.0, 0.027),
]


def _state(case, k, measure=False):
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA
    from cudapic_b200.workloads import steady_state
    n_g, ne, ni, v, p, gap = case
    params = cp.default_params(voltage=v, pressure=p, gap=gap, n_g=n_g, capacity=2048, weight=7.0e4)
    st = GpuSimState(params)
    g = st.grid
    e = steady_state(ne, E_MASS, 3.0, gap=gap, dt=g.dt_e, seed=100 + k)
    i = steady_state(ni, AR_MASS, 0.03, gap=gap, dt=g.dt_i, seed=200 + k)
    st.upload_electrons(ParticlesSoA(*e))
    st.upload_ions(ParticlesSoA(*i))
    st.seed(e_master=(0x1234 + k, 0x11112222, 0x22223333, 0x33334444),
            i_master=(0x4444 + k, 0x55556666, 0x66667777, 0x77778888))
    if measure:
        st.set_measure(True)
    return st


def _plane(ptr, n, dtype):
    from gpu_util import device_array
    return device_array(ptr, n, dtype)


def _snapshot(st):
    """Counts, sorted particle rows, RNG planes, field and densities of a state."""
    from gpu_util import sorted_rows
    st.synchronize()
    ne, ni = st.counts()
    e, _ = st.download_electrons()
    i, _ = st.download_ions()
    b = st.buffers()
    cap, n_g = st.capacity, st.grid.n_g
    rng = [_plane(b.rng[sp][k], cap, np.uint32) for sp in (0, 1) for k in range(4)]
    return {
        "counts": (ne, ni),
        "e": sorted_rows(e.x, e.vx, e.vy, e.vz),
        "i": sorted_rows(i.x, i.vx, i.vy, i.vz),
        "rng": rng,
        "efield": _plane(b.efield, n_g, np.float32),
        "pot": _plane(b.pot, n_g, np.float32),
        "e_density": _plane(b.e_density, n_g, np.float32),
        "i_density": _plane(b.i_density, n_g, np.float32),
        "work": st.work(),
        "err": st.device_error(),
    }


def _compare(a, b, label):
    assert a["err"] == 0 and b["err"] == 0, label
    assert a["counts"] == b["counts"], label
    np.testing.assert_array_equal(a["e"], b["e"], err_msg=label)
    for k, (ra, rb) in enumerate(zip(a["rng"][:4], b["rng"][:4])):
        np.testing.assert_array_equal(ra, rb, err_msg="%s electron rng plane %d" % (label, k))
    # Ions: positions exactly.  Ions spawned by this step's ionizations take
    # their slots in claim order, which no launch fixes, and the ion
    # collision test that follows draws from the stream of that slot; so the
    # velocities and RNG states of those few ions may differ between runs.
    np.testing.assert_array_equal(a["i"][:, 0], b["i"][:, 0], err_msg=label)
    spawned_bound = max(4, a["i"].shape[0] // 100)
    assert np.count_nonzero(np.any(a["i"] != b["i"], axis=1)) <= spawned_bound, label
    diff = np.zeros(a["rng"][4].shape[0], bool)
    for ra, rb in zip(a["rng"][4:], b["rng"][4:]):
        diff |= ra != rb
    assert np.count_nonzero(diff) <= spawned_bound, label
    np.testing.assert_array_equal(a["efield"], b["efield"], err_msg=label)
    np.testing.assert_array_equal(a["pot"], b["pot"], err_msg=label)
    # next-step densities: the same fixed-point node sums, added across CTAs
    # in f32 (different partitions round the f32 additions differently)
    for key in ("e_density", "i_density"):
        scale = max(1.0, float(np.abs(b[key]).max()))
        np.testing.assert_allclose(a[key], b[key], rtol=0, atol=2e-6 * scale, err_msg="%s %s" % (label, key))
    assert a["work"] == b["work"], label


def test_batch_first_step_bit_exact_against_each_discharge_alone(cudapic, cuda_device):
    """One step (an ion step: Poisson, ion push, fused electron step, ion
    collisions) of a batch of ragged discharges equals, per discharge, the
    same step of the fused driver alone: same survivors, spawns and RNG
    streams bit for bit."""
    from cudapic_b200.sim import GpuBatch
    together = [_state(c, k) for k, c in enumerate(CASES)]
    alone = [_state(c, k) for k, c in enumerate(CASES)]
    try:
        with GpuBatch(together) as b:
            b.run_steps(1)
            b.synchronize()
        for st in alone:
            st.run_steps(1)
        for k, (x, y) in enumerate(zip(together, alone)):
            _compare(_snapshot(x), _snapshot(y), "discharge %d" % k)
            assert x.steps_done() == y.steps_done() == 1
    finally:
        for st in together + alone:
            st.close()


def test_batch_measurements_match_each_discharge_alone(cudapic, cuda_device):
    """The measurement window of a batched step (electrode counters and
    IFEDs, collision counts, time-averaged densities, EEPF) equals the
    discharges' own."""
    from cudapic_b200.sim import GpuBatch
    together = [_state(c, k, measure=True) for k, c in enumerate(CASES)]
    alone = [_state(c, k, measure=True) for k, c in enumerate(CASES)]
    try:
        with GpuBatch(together) as b:
            b.run_steps(1)
            b.synchronize()
        for st in alone:
            st.run_steps(1)
        for k, (x, y) in enumerate(zip(together, alone)):
            wx, wy = x.wall_counters(), y.wall_counters()
            for sp in ("e", "i"):
                for key in ("abs_pow", "abs_gnd"):
                    assert wx[sp][key] == wy[sp][key], (k, sp, key)
                for key in ("ifed_pow", "ifed_gnd"):
                    np.testing.assert_array_equal(np.asarray(wx[sp][key]), np.asarray(wy[sp][key]))
            cx, cy = x.download_measurements(), y.download_measurements()
            for a, c in zip(cx, cy):
                np.testing.assert_array_equal(np.asarray(a), np.asarray(c))
            rx, ry = x.report(), y.report()
            assert rx["steps_measured"] == ry["steps_measured"] == 1
            np.testing.assert_equal(rx["e_coll_freq"], ry["e_coll_freq"])  # NaN without electrons
            # ion collisions: exact up to the ions spawned this step (their
            # slots, hence their RNG streams, follow the claim order)
            n_i = x.counts()[1]
            dt = x.grid.dt_e
            cx_i, cy_i = rx["i_coll_freq"] * dt * n_i, ry["i_coll_freq"] * dt * n_i
            assert not (abs(cx_i - cy_i) > 4.5), (k, cx_i, cy_i)
            if ry["mean_energy_center"] == ry["mean_energy_center"]:  # not NaN
                assert rx["mean_energy_center"] == pytest.approx(ry["mean_energy_center"], rel=1e-12)
    finally:
        for st in together + alone:
            st.close()


def test_batch_runs_graphs_and_tracks_its_states(cudapic, cuda_device):
    """Graph-captured periods (2 N_SUB steps) and single steps mixed; the
    states' own calls work between batch runs; stepping a state on its own
    stops the batch until the others catch up, and the batch then rebuilds
    its descriptors for the moved buffers."""
    from cudapic_b200 import CudapicError
    from cudapic_b200.sim import GpuBatch
    states = [_state(c, k) for k, c in enumerate(CASES)]
    try:
        with GpuBatch(states) as b:
            b.run_steps(3)       # three single steps
            b.run_steps(37)      # up to the period boundary
            b.run_steps(80)      # two captured periods
            b.synchronize()
            n1 = [st.counts() for st in states]
            w1 = [st.work() for st in states]
            assert [st.steps_done() for st in states] == [120] * len(states)
            assert all(st.device_error() == 0 for st in states)
            for (ne, ni), c in zip(n1, CASES):
                if c[1] >= 500:
                    assert 0.5 * c[1] < ne < 2 * c[1]
                assert ni > 0
            # work: electrons every step, ions on 6 of the 120 steps
            for w, (ne, ni) in zip(w1, n1):
                assert w > 0
            states[0].run_steps(1)
            with pytest.raises(CudapicError):
                b.run_steps(1)
            for st in states[1:]:
                st.run_steps(1)
            b.run_steps(40)
            b.synchronize()
            assert [st.steps_done() for st in states] == [161] * len(states)
            assert all(st.device_error() == 0 for st in states)
            for st in states:
                e, _ = st.download_electrons()
                assert np.all((e.x >= 0) & (e.x <= st.params.gap))
    finally:
        for st in states:
            st.close()


def test_batch_agrees_with_discharges_alone_over_a_period(cudapic, cuda_device):
    """Over two graph periods (80 steps) the batched discharges
    stay statistically with the same discharges run alone (the runs diverge
    after the first step only through compaction order)."""
    from cudapic_b200.sim import GpuBatch
    cases = [c for c in CASES if c[1] >= 600]
    together = [_state(c, k) for k, c in enumerate(cases)]
    alone = [_state(c, k) for k, c in enumerate(cases)]
    try:
        with GpuBatch(together) as b:
            b.run_steps(80)
            b.synchronize()
        for st in alone:
            st.run_steps(80)
        for x, y in zip(together, alone):
            (ex, ix), (ey, iy) = x.counts(), y.counts()
            assert abs(ex - ey) <= 0.03 * ey + 10
            assert abs(ix - iy) <= 0.03 * iy + 10
            vx, _ = x.download_electrons()
            vy, _ = y.download_electrons()
            kx = np.mean(vx.vx.astype(np.float64) ** 2 + vx.vy ** 2 + vx.vz ** 2)
            ky = np.mean(vy.vx.astype(np.float64) ** 2 + vy.vy ** 2 + vy.vz ** 2)
            assert kx == pytest.approx(ky, rel=0.1)
    finally:
        for st in together + alone:
            st.close()


def test_batch_class_steps_every_discharge(cudapic, cuda_device):
    from cudapic_b200.batch import Batch, c2_specs
    specs = c2_specs(n=6, seed=7)
    for s in specs:
        s.particles = min(s.particles, 40_000)
    with Batch(specs) as b:
        n0 = b.counts()
        t, w = b.timed_steps(120)
        assert t > 0 and w > 0
        assert w == b.work()                       # nothing ran before the timed steps
        n1 = b.counts()
        assert all(e == 0 for e in b.device_errors())
        for (e0, i0), (e1, i1), s in zip(n0, n1, specs):
            assert (e0, i0) == (s.particles, s.particles)
            assert 0 < e1 < 2 * s.particles and 0 < i1 < 2 * s.particles
        assert 120 * min(e for e, _ in n1) <= w
        assert [st.steps_done() for st in b.states] == [120] * len(specs)


def test_batch_spawns_stay_with_their_discharge(cudapic, cuda_device):
    """Strongly ionizing discharges of ragged sizes in one batch, so that
    warps of the batched scatter pass straddle two discharges while both
    ionize: over 38 in-place steps (two compacting ones) every discharge's
    electron and ion counts stay with the same discharge run alone (each
    spawn claims a slot of its own discharge's counter), and no capacity
    is exceeded."""
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuBatch, GpuSimState, ParticlesSoA
    from cudapic_b200.workloads import steady_state
    sizes = [1203, 2999, 517, 4001, 1777, 3333, 901, 2500]

    def make(k, n):
        params = cp.default_params(voltage=480.0, pressure=40.0, gap=0.025, n_g=400, capacity=16384,
                                   weight=7.0e4)
        st = GpuSimState(params)
        g = st.grid
        st.upload_electrons(ParticlesSoA(*steady_state(n, E_MASS, 20.0, gap=0.025, dt=g.dt_e, seed=300 + k)))
        st.upload_ions(ParticlesSoA(*steady_state(n, AR_MASS, 0.03, gap=0.025, dt=g.dt_i, seed=400 + k)))
        st.seed(e_master=(0x5151 + k, 0x11112222, 0x22223333, 0x33334444),
                i_master=(0x6161 + k, 0x55556666, 0x66667777, 0x77778888))
        return st

    together = [make(k, n) for k, n in enumerate(sizes)]
    alone = [make(k, n) for k, n in enumerate(sizes)]
    try:
        with GpuBatch(together) as b:
            b.run_steps(40)
            b.synchronize()
        for st in alone:
            st.run_steps(40)
        grew = 0
        for k, (x, y) in enumerate(zip(together, alone)):
            assert x.device_error() == 0 and y.device_error() == 0, k
            (ex, ix), (ey, iy) = x.counts(), y.counts()
            grew += ix > sizes[k] + 20  # ions: spawned by ionizations, barely absorbed in two ion steps
            assert abs(ex - ey) <= 0.05 * ey + 20, (k, ex, ey)
            assert abs(ix - iy) <= 0.05 * iy + 20, (k, ix, iy)
        assert grew == len(sizes)  # every discharge ionizes
    finally:
        for st in together + alone:
            st.close()
