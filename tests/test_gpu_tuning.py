"""GPU tests: every launch shape the tuner may pick keeps the kernels exact
(bit-exact survivors and collision outcomes, deposit within tolerance)."""
import numpy as np
import pytest

from gpu_util import check_step_electrons, counter, dev, host, sorted_rows, zeros

pytestmark = pytest.mark.gpu

E_MASS = 9.10938356e-31

SHAPES = [
    dict(density_threads=256, density_ctas_per_sm=1, density_copies=2, density_cluster=1, push_stages=2,
         push_ctas_per_sm=1, mcc_stages=2, mcc_ctas_per_sm=1, mcc_variant=2, step_rows=2, step_stages=2,
         step_ctas_per_sm=1),
    dict(density_threads=1024, density_ctas_per_sm=4, density_copies=32, density_cluster=8, push_stages=6,
         push_ctas_per_sm=2, mcc_stages=4, mcc_ctas_per_sm=2, mcc_variant=2, step_rows=4, step_stages=6,
         step_ctas_per_sm=4),
    dict(density_threads=512, density_ctas_per_sm=2, density_copies=8, density_cluster=2, push_stages=5,
         push_ctas_per_sm=3, mcc_stages=3, mcc_ctas_per_sm=3, mcc_variant=1, step_rows=2, step_stages=5,
         step_ctas_per_sm=3),
]


@pytest.fixture
def restore_tuning(cudapic):
    saved = cudapic.get_tuning()
    yield
    cudapic.set_tuning(**saved)


@pytest.mark.parametrize("shape", range(len(SHAPES)))
def test_kernels_exact_under_every_shape(cudapic, oracle, tables, cuda_device, restore_tuning, shape):
    from cudapic_b200.workloads import field_profile, steady_state
    cudapic.set_tuning(**SHAPES[shape])
    K = cudapic.kernels
    n = 150_001
    cap = (n + n // 2 + 3) // 4 * 4
    g = cudapic.grid_from_params(capacity=cap, n_t=400)
    ph = oracle.phys_from_params(capacity=cap, n_t=400)
    x, vx, vy, vz = steady_state(n, E_MASS, 15.0, dt=g.dt_e, seed=shape)

    dens = zeros(400)
    K.get_density(dev(x), dens, counter(n), g)
    ref = oracle.get_density_f64(x, ph)
    assert np.linalg.norm(host(dens) - ref) / np.linalg.norm(ref) < 3e-5

    ef = field_profile(400)
    pad = lambda a, t=np.float32: np.concatenate([a, np.zeros(cap - len(a), t)])  # noqa: E731
    src = [dev(pad(a)) for a in (x, vx, vy, vz)]
    dst = [zeros(cap) for _ in range(4)]
    alive = counter(0)
    K.move_and_compact(dev(ef), *src, *dst, alive, counter(n), g.factor_e, g.dt_e, g)
    m = int(host(alive)[0])
    rx = oracle.move_and_compact(ef, x, vx, vy, vz, g.factor_e, g.dt_e, ph)
    assert m == rx[0].size
    assert np.array_equal(sorted_rows(*[host(d)[:m] for d in dst]), sorted_rows(*rx[:4]))

    cs, se, si = tables
    e_h = [pad(a) for a in (x, vx, vy, vz)]
    i_h = [np.zeros(cap, np.float32) for _ in range(4)]
    r_h = [pad(np.asarray(p), np.uint32) for p in oracle.seed_streams([2, 7, 1, 8], n)]
    e_d, i_d, r_d = [dev(a) for a in e_h], [dev(a) for a in i_h], [dev(a) for a in r_h]
    ev = zeros(n, np.uint8)
    ae, ai = counter(n), counter(0)
    K.check_collisions_e(dev(se), dev(cs), counter(n), *e_d, *r_d, *i_d, ae, ai, g, events=ev)
    ev_ref, ne_ref, ni_ref, _ = oracle.check_collisions_e(se, cs, n, e_h, r_h, i_h, n, 0, ph)
    assert np.array_equal(host(ev), ev_ref)
    assert (ev_ref > 0).sum() > 100
    assert int(host(ae)[0]) == ne_ref and int(host(ai)[0]) == ni_ref
    for d, h in zip(r_d, r_h):
        assert np.array_equal(host(d)[:n], h[:n])

    # the fused electron step under the same shape
    dev_tables = (dev(cs), dev(se), dev(si))
    cap2 = (2 * n + 4096 + 3) // 4 * 4
    g2 = cudapic.grid_from_params(capacity=cap2, n_t=100)
    ph2 = oracle.phys_from_params(capacity=cap2, n_t=100)
    check_step_electrons(K, oracle, tables, dev_tables, g2, ph2, x, vx, vy, vz, ef, cap2)


INPLACE_SHAPES = [
    dict(inplace_copies=-1, inplace_ctas_per_sm=4, inplace_prefetch=1, scatter_ctas_per_sm=4),
    dict(inplace_copies=1, inplace_ctas_per_sm=2, inplace_prefetch=-1, scatter_ctas_per_sm=1),
    dict(inplace_copies=4, inplace_ctas_per_sm=3, inplace_prefetch=3, scatter_ctas_per_sm=8),
]


@pytest.mark.parametrize("shape", range(len(INPLACE_SHAPES)))
def test_inplace_step_exact_under_every_shape(cudapic, oracle, tables, cuda_device, restore_tuning, shape):
    """The in-place electron step (stream + scatter pass) under the
    in-place launch shapes the tuner may pick: f32 or fixed-point
    histograms, CTAs per SM, L2 prefetch distance, scatter CTAs per SM --
    slots, RNG states and spawns bit-exact, density within the deposit
    tolerance of the f32 histogram."""
    from cudapic_b200.workloads import field_profile, steady_state
    from gpu_util import check_step_inplace, dead_mask
    cudapic.set_tuning(**INPLACE_SHAPES[shape])
    cs, se, si = tables
    dev_tables = (dev(cs), dev(se), dev(si))
    n = 300_001
    cap = (2 * n + 4096 + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=100, capacity=cap)
    ph = oracle.phys_from_params(n_t=100, capacity=cap)
    x, vx, vy, vz = steady_state(n, E_MASS, 30.0, dt=g.dt_e, seed=40 + shape)
    m, ne, ni, nc = check_step_inplace(K=cudapic.kernels, oracle=oracle, tables=tables, dev_tables=dev_tables,
                                       g=g, ph=ph, x=x, vx=vx, vy=vy, vz=vz, ef=field_profile(400), cap=cap,
                                       dead=dead_mask(n, 0.02), dens_tol=max(2e-5, 1.5 * 400 * 2.0 ** -24))
    assert nc > 1000 and ne > n
