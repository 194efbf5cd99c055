"""GPU tests of the XT diagnostics and the <j E> power absorption (eduPIC's
measurement mode, C/eduPIC.cc:557-614, :705-715, :864-903, :1011-1026)
against the oracle's restatement of one step and of norm_all_xt."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26
E_CHARGE = 1.60217662e-19


def _state(n, n_g=400, seed=3, **kw):
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA
    from cudapic_b200.workloads import steady_state
    params = cp.default_params(n_g=n_g, capacity=2 * n, weight=7.0e4 * 120000 / n, **kw)
    st = GpuSimState(params)
    g = st.grid
    e = steady_state(n, E_MASS, 3.0, gap=params.gap, dt=g.dt_e, seed=seed)
    i = steady_state(n, AR_MASS, 0.03, gap=params.gap, dt=g.dt_i, seed=seed + 1)
    st.upload_electrons(ParticlesSoA(*e))
    st.upload_ions(ParticlesSoA(*i))
    st.seed()
    return st, e, i


def test_xt_first_step_matches_oracle(cudapic, cuda_device, oracle, tables):
    """Step 0 (an ion step) of a measurement window: column 0 of every XT
    quantity equals the oracle's accumulation of the particles before the
    push in the step's field, normalised as eduPIC does (f32 partial sums
    per CTA, hence the 2e-5 relative tolerance); the other columns are 0."""
    from gpu_util import device_array
    n = 60_000
    st, e, i = _state(n)
    try:
        st.set_measure(True)
        st.run_steps(1)
        st.synchronize()
        n_g, n_xt = st.xt_shape()
        assert (n_g, n_xt) == (400, 200)
        b = st.buffers()
        ef = device_array(b.efield, n_g, np.float32)
        pot = device_array(b.pot, n_g, np.float32)
        cumul_e, cumul_i, _ = st.download_measurements()
        ph = oracle.phys_from_params(capacity=2 * n, weight=7.0e4 * 120000 / n)
        cs_ion = tables[0].reshape(5, -1)[2]
        re = oracle.xt_accumulate(ef, *e, False, cs_ion, ph)
        ri = oracle.xt_accumulate(ef, *i, True, None, ph)
        raw = {"count_e": re[0], "ue": re[1], "meanee": re[2], "ioniz": re[3], "count_i": ri[0], "ui": ri[1],
               "meanei": ri[2], "pot": pot.astype(np.float64), "efield": ef.astype(np.float64),
               "ne": np.asarray(cumul_e), "ni": np.asarray(cumul_i)}
        raw = {k: np.stack([v] + [np.zeros_like(v)] * (n_xt - 1), axis=1) for k, v in raw.items()}
        p = st.params
        want = oracle.xt_normalise(raw, p.n_t, n_xt, 1, p.gap, p.n_g, p.frequency, p.weight, p.electrode_area)
        for name in ("pot", "efield", "ne", "ni"):
            np.testing.assert_array_equal(st.download_xt(name), want[name], err_msg=name)
        for name in ("je", "ji", "powere", "poweri", "meanee", "meanei", "ioniz"):
            got = st.download_xt(name)
            scale = float(np.abs(want[name]).max())
            assert scale > 0, name
            np.testing.assert_allclose(got, want[name], rtol=2e-5, atol=2e-5 * scale, err_msg=name)
            assert not np.any(got[:, 1:]), name
    finally:
        st.close()


def test_xt_batched_step_matches_each_discharge_alone(cudapic, cuda_device):
    """A measuring batch fills every discharge's XT columns like the
    discharges alone (same first step; f32 partial sums per CTA differ in
    partition, hence the tolerance)."""
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuBatch, GpuSimState, ParticlesSoA
    from cudapic_b200.workloads import steady_state
    cases = [(400, 1500, 250.0, 10.0, 0.025), (200, 997, 120.0, 30.0, 0.018), (800, 1789, 480.0, 6.0, 0.038)]

    def make(k, case):
        n_g, n, v, p, gap = case
        st = GpuSimState(cp.default_params(voltage=v, pressure=p, gap=gap, n_g=n_g, capacity=2048, weight=7.0e4))
        g = st.grid
        st.upload_electrons(ParticlesSoA(*steady_state(n, E_MASS, 3.0, gap=gap, dt=g.dt_e, seed=10 + k)))
        st.upload_ions(ParticlesSoA(*steady_state(n, AR_MASS, 0.03, gap=gap, dt=g.dt_i, seed=20 + k)))
        st.seed(e_master=(0x1234 + k, 1, 2, 3), i_master=(0x4444 + k, 5, 6, 7))
        st.set_measure(True)
        return st

    together = [make(k, c) for k, c in enumerate(cases)]
    alone = [make(k, c) for k, c in enumerate(cases)]
    try:
        with GpuBatch(together) as b:
            b.run_steps(1)
            b.synchronize()
        for st in alone:
            st.run_steps(1)
        for k, (x, y) in enumerate(zip(together, alone)):
            for name in ("pot", "efield", "ne", "ni"):
                np.testing.assert_array_equal(x.download_xt(name), y.download_xt(name), err_msg="%d %s" % (k, name))
            for name in ("je", "ji", "meanee", "meanei", "ioniz", "powere", "poweri"):
                gx, gy = x.download_xt(name), y.download_xt(name)
                scale = max(1e-300, float(np.abs(gy).max()))
                np.testing.assert_allclose(gx, gy, rtol=2e-5, atol=2e-5 * scale, err_msg="%d %s" % (k, name))
    finally:
        for st in together + alone:
            st.close()


def test_xt_files_and_power_over_periods(cudapic, cuda_device, tmp_path):
    """Two RF periods of measurement: every column filled, eduPIC's eleven
    *_xt.dat files of N_G rows and N_XT columns, and the report's <j E>
    power: the electrons absorb power on average, and the space-time mean
    of the power files is the report's figure."""
    st, _, _ = _state(200_000)
    try:
        st.run_steps(4000)
        st.set_measure(True)
        st.run_steps(8000)
        st.synchronize()
        n_g, n_xt = st.xt_shape()
        ne = st.download_xt("ne")
        assert np.all(ne[n_g // 2] > 0)                     # the centre is populated in every column
        st.write_xt(tmp_path)
        for name in ("pot", "efield", "ne", "ni", "je", "ji", "powere", "poweri", "meanee", "meanei", "ioniz"):
            a = np.loadtxt(tmp_path / ("%s_xt.dat" % name))
            assert a.shape == (n_g, n_xt), name
            np.testing.assert_allclose(a, st.download_xt(name), rtol=2e-6, atol=1e-300)
        r = st.report()
        assert r["power_e"] > 0 and np.isfinite(r["power_i"])
        assert r["power_e"] == pytest.approx(float(st.download_xt("powere").mean()), rel=1e-12)
        assert r["power_i"] == pytest.approx(float(st.download_xt("poweri").mean()), rel=1e-12)
        st.write_info(tmp_path / "info.txt")
        text = (tmp_path / "info.txt").read_text()
        if r["conditions_ok"]:
            assert "Absorbed power calculated as <j*E>:" in text
    finally:
        st.close()
