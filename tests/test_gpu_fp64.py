"""GPU tests of the all-FP64 twin (cudapic_fp64_*): exact window sums
(the boundary potential is the RF table, the deposit conserves the
particles' weight), and the twin against the f32 driver over 400 steps from
the same particles and RNG streams (statistically the same discharge)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26


def _state(n=20000, seed=3):
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA
    from cudapic_b200.workloads import steady_state
    st = GpuSimState(cp.default_params(capacity=4 * n, weight=7e4 * 120000 / n))
    g = st.grid
    st.upload_electrons(ParticlesSoA(*steady_state(n, E_MASS, 3.0, dt=g.dt_e, seed=seed)))
    st.upload_ions(ParticlesSoA(*steady_state(n, AR_MASS, 0.03, dt=g.dt_i, seed=seed + 1)))
    st.seed(e_master=(0x1234 + seed, 0x11112222, 0x22223333, 0x33334444),
            i_master=(0x4444 + seed, 0x55556666, 0x66667777, 0x77778888))
    return st


def test_fp64_window_sums_are_exact(cudapic, cuda_device):
    """One measured step: the electron density integrates (trapezoid, the
    doubled boundary nodes halved again) to the electrons' weight; over two
    more steps (1 .. 39) the potential at the powered electrode sums the RF values of
    those steps and the grounded one stays zero."""
    from cudapic_b200.fp64 import Fp64Discharge
    st = _state()
    try:
        n_e, _ = st.counts()
        p = st.params
        dx = p.gap / (p.n_g - 1)
        with Fp64Discharge(st) as tw:
            tw.set_measure(True)
            tw.run_steps(1)
            m = tw.measurements()
            integral = (m["cumul_e"].sum() - 0.5 * (m["cumul_e"][0] + m["cumul_e"][-1])) * dx
            assert integral * p.electrode_area / p.weight == pytest.approx(n_e, rel=1e-12)
            tw.set_measure(True)
            tw.run_steps(39)
            m = tw.measurements()
            assert (m["steps"], m["ion_steps"]) == (39, 1)  # steps 1 .. 39: the ion step 20
            t = np.arange(1, 40)
            rf = p.voltage * np.cos(t / p.n_t * 2 * np.pi)
            assert m["pot_sum"][0] == pytest.approx(rf.sum(), rel=1e-12, abs=1e-9)
            assert m["pot_sum"][-1] == 0.0
            assert m["device_error"] == 0
    finally:
        st.close()


def test_fp64_twin_tracks_the_f32_driver(cudapic, cuda_device):
    """400 steps from the same particles and streams: counts within 3 % (+10),
    every electron of the f32 run inside the gap, no device errors."""
    from cudapic_b200.fp64 import Fp64Discharge
    st = _state()
    try:
        with Fp64Discharge(st) as tw:
            tw.run_steps(400)
            m = tw.measurements()
            st.run_steps(400)
            ne, ni = st.counts()
            e, _ = st.download_electrons()
        for a, b in zip(m["counts"], (ne, ni)):
            assert abs(a - b) <= 0.03 * b + 10, (m["counts"], (ne, ni))
        assert m["device_error"] == 0 and st.device_error() == 0
        assert np.all((e.x >= 0) & (e.x <= st.params.gap))
    finally:
        st.close()
