"""The ion test's certain-rejection bound (mcc.cuh ion_collides, the
bounded ion MCC entry) checked on the CPU against the oracle's full test
(Rust-CUDA/src/main.rs:1180-1197): no ion whose test draw lies at or above
the bound collides, over populations from thermal to 20 eV ions and time
steps up to 200x the reference's.  The draws are xoshiro128+ steps restated
in numpy (the fifth output of each slot's stream: four for the target's
Box-Muller normals, then the test draw)."""
import numpy as np
import pytest

AR_MASS = 6.63352090e-26


def _next(s):
    """One xoshiro128+ step of every stream (four uint32 planes, updated in place)."""
    s0, s1, s2, s3 = s
    out = (s0 + s3).astype(np.uint32)
    t = (s1 << np.uint32(9)).astype(np.uint32)
    s2 ^= s0
    s3 ^= s1
    s1 ^= s2
    s0 ^= s3
    s2 ^= t
    s3[:] = ((s3 << np.uint32(11)) | (s3 >> np.uint32(21))).astype(np.uint32)
    return out


def _uniform(out):
    return ((out >> np.uint32(9)) | np.uint32(0x3F800000)).view(np.float32) - np.float32(1.0)


def _bound(k, vx, vy, vz, normal_range):
    """fmaf(k, |v| + 9.2 sigma, 6e-7) as the kernels compute it (f32 inputs,
    one rounding of the fused multiply-add)."""
    v2 = (vx * vx + vy * vy + vz * vz).astype(np.float32)
    vmag = np.sqrt(v2).astype(np.float32)
    s = (vmag + np.float32(9.2) * np.float32(normal_range)).astype(np.float32)
    return (np.float64(k) * s.astype(np.float64) + 6e-7).astype(np.float32)


@pytest.mark.parametrize("n_t,temp,seed", [(4000, 0.03, 1), (4000, 2.0, 2), (200, 0.03, 3), (200, 20.0, 4),
                                           (20, 2.0, 5), (20, 20.0, 6)])
def test_no_ion_above_the_bound_collides(cudapic, oracle, tables, n_t, temp, seed):
    from cudapic_b200.workloads import steady_state
    cs, _, si = tables
    n = 200_000
    g = cudapic.grid_from_params(n_t=n_t, capacity=n)
    ph = oracle.phys_from_params(n_t=n_t, capacity=n)
    k = np.nextafter(np.float32(float(si.max()) * float(g.dt_i) * (1.0 + 1e-5)), np.float32(np.inf))
    _, vx, vy, vz = steady_state(n, AR_MASS, temp, seed=seed, edge_fraction=0.0)
    rng = [np.asarray(p).copy() for p in oracle.seed_streams([seed, 7, 11, 13], n)]
    s = [p.copy() for p in rng]
    for _ in range(4):
        _next(s)
    u = _uniform(_next(s))
    b = _bound(k, vx, vy, vz, g.normal_range)
    events = oracle.check_collisions_i(si, cs, n, [vx.copy(), vy.copy(), vz.copy()], [p.copy() for p in rng], ph)
    skipped = u >= b
    assert not np.any(events[skipped]), "an ion above the bound collided"
    assert np.any(events > 0)
    if n_t == 4000:  # the reference's time step: nearly every ion skips the target's transcendentals
        assert skipped.mean() > 0.9, skipped.mean()
