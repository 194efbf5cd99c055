"""CPU tests of the oracle's voltage-sensitivity model: the pathwise adjoint
(collision events and random draws frozen) against central differences of
the same deterministic model, the f32 model of the CUDA path against the
double one, the horizon option."""
import numpy as np
import pytest

E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26


def _case(oracle, n=2000, seed=1):
    from cudapic_b200.workloads import steady_state
    cap = 2 * n + 1000
    ph = oracle.phys_from_params(capacity=cap, weight=7e4 * 120000 / n)
    e = steady_state(n, E_MASS, 3.0, dt=ph.dt_e, seed=seed)
    i = steady_state(n, AR_MASS, 0.03, dt=ph.dt_i, seed=seed + 1)
    st = oracle.SensState(cap, e, i, oracle.seed_streams([1, 2, 3, 4], cap), oracle.seed_streams([5, 6, 7, 8], cap))
    return ph, st


def test_adjoint_matches_central_difference(oracle, tables):
    """Double model, 100 steps: the adjoint equals the derivative of the
    same deterministic run (central differences at dV = 1 mV keep every
    collision decision and absorption of the run) to 1e-4."""
    ph, st0 = _case(oracle)
    obs, grad = oracle.sens_run(ph, tables, 250.0, 100, st0.copy(), f64=True)
    h = 1e-3
    up, _ = oracle.sens_run(ph, tables, 250.0 + h, 100, st0.copy(), f64=True, grad=False)
    dn, _ = oracle.sens_run(ph, tables, 250.0 - h, 100, st0.copy(), f64=True, grad=False)
    for k in range(2):
        fd = (up[k] - dn[k]) / (2 * h)
        assert grad[k] == pytest.approx(fd, rel=1e-4), (k, grad[k], fd)
    assert obs[0] != 0.0 and obs[1] > 0.0


def test_f32_model_adjoint_agrees_with_double_model(oracle, tables):
    """The f32 arithmetic of the CUDA path and the double model give the same
    derivative over a short window (their trajectories differ by rounding)."""
    ph, st0 = _case(oracle)
    o32, g32 = oracle.sens_run(ph, tables, 250.0, 100, st0.copy(), f64=False)
    o64, g64 = oracle.sens_run(ph, tables, 250.0, 100, st0.copy(), f64=True)
    for k in range(2):
        assert o32[k] == pytest.approx(o64[k], rel=1e-3)
        assert g32[k] == pytest.approx(g64[k], rel=1e-3)


def test_horizon(oracle, tables):
    """A horizon equal to the window is the full adjoint; a shorter one
    truncates the voltage's influence (the flux of ions, which move every
    N_SUB steps, loses its history entirely at horizon N_SUB)."""
    ph, st0 = _case(oracle)
    _, g0 = oracle.sens_run(ph, tables, 250.0, 100, st0.copy(), horizon=0)
    _, gk = oracle.sens_run(ph, tables, 250.0, 100, st0.copy(), horizon=100)
    _, g20 = oracle.sens_run(ph, tables, 250.0, 100, st0.copy(), horizon=20)
    assert g0 == gk
    assert g20[1] == 0.0 and g20[0] != g0[0]
    with pytest.raises(ValueError):
        oracle.sens_run(ph, tables, 250.0, 100, st0.copy(), horizon=30)


def test_slot_form_keeps_slots_and_appends_spawns(oracle, tables):
    """Absorbed particles stay dead in their slots, live ones stay inside the
    gap, and the spawns of a run fill the slots after the initial count."""
    ph, st0 = _case(oracle)
    s = st0.copy()
    oracle.sens_run(ph, tables, 250.0, 200, s, grad=False)
    for k in range(2):
        x = s.p[k][0][:s.n[k]]
        dead = x < 0
        assert np.all(x[dead] == -1.0)
        assert np.all((x[~dead] >= 0) & (x[~dead] <= ph.gap))
        assert s.n[k] > st0.n[k]          # ionizations appended children
        assert dead.sum() > 0             # and some particles reached the electrodes
    assert s.n[0] - st0.n[0] == s.n[1] - st0.n[1]
    assert s.dev_err == 0


@pytest.mark.parametrize("n_g", [3, 4, 57, 400, 4096])
def test_poisson_adjoint_is_the_transpose(oracle, n_g):
    """<eb, E(dn_e, dn_i, dpot0)> = <neb, dn_e> + <nib, dn_i> + pot0b dpot0
    for the FP64 solve (linear with zero base), random vectors."""
    ph = oracle.phys_from_params(n_g=n_g)
    rng = np.random.default_rng(n_g)
    eb = rng.normal(size=n_g)
    neb, nib, p0b = oracle.sens_poisson_adjoint(eb, ph)
    for _ in range(3):
        dne = rng.normal(size=n_g).astype(np.float32) * np.float32(1e15)
        dni = rng.normal(size=n_g).astype(np.float32) * np.float32(1e15)
        dp0 = float(rng.normal() * 100.0)
        ef = oracle.poisson_thomas_f64(dne, dni, dp0, ph)[1]
        lhs = float(np.dot(eb, ef))
        rhs = float(np.dot(neb, dne.astype(np.float64)) + np.dot(nib, dni.astype(np.float64)) + p0b * dp0)
        assert lhs == pytest.approx(rhs, rel=1e-9, abs=1e-9 * np.abs(eb).sum() * np.abs(ef).max())


def test_spawns_beyond_capacity_are_dropped_and_flagged(oracle, tables):
    """A capacity just above the initial counts: the spawns that find no slot
    are dropped, both counts stop at the capacity, both error bits are set."""
    from cudapic_b200.workloads import steady_state
    n = 2000
    cap = n + 8
    ph = oracle.phys_from_params(capacity=cap, weight=7e4 * 120000 / n)
    e = steady_state(n, E_MASS, 12.0, dt=ph.dt_e, seed=4)
    i = steady_state(n, AR_MASS, 0.03, dt=ph.dt_i, seed=5)
    st = oracle.SensState(cap, e, i, oracle.seed_streams([1, 2, 3, 4], cap), oracle.seed_streams([5, 6, 7, 8], cap))
    obs, grad = oracle.sens_run(ph, tables, 250.0, 200, st)
    assert st.n == [cap, cap]
    assert st.dev_err == 0x3
    assert np.isfinite(obs).all() and np.isfinite(grad).all()


def test_study_summary_statistics(cudapic):
    """The study's per-start aggregation: mean and standard error."""
    from cudapic_b200.sensitivity import mean_and_error
    m, e = mean_and_error([1.0, 2.0, 3.0, 6.0])
    assert m == 3.0 and e == pytest.approx(np.std([1.0, 2.0, 3.0, 6.0], ddof=1) / 2.0)
    m, e = mean_and_error([4.0])
    assert m == 4.0 and e != e  # NaN: no spread from one start
