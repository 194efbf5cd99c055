"""GPU tests of the batched path: independent discharges on their own
streams step correctly side by side."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_specs(n=6):
    from cudapic_b200.batch import c2_specs
    specs = c2_specs(n=n, seed=7)
    for s in specs:
        s.particles = min(s.particles, 40_000)
    return specs


def test_batch_steps_every_discharge(cudapic, cuda_device):
    from cudapic_b200.batch import Batch
    specs = _small_specs()
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
        # particle-steps: electrons every step, ions on every 20th (6 of 120)
        assert 120 * min(e for e, _ in n1) <= w
        assert [st.steps_done() for st in b.states] == [120] * len(specs)


def test_batch_discharge_matches_the_same_discharge_alone(cudapic, cuda_device):
    """A discharge inside a batch evolves like the same discharge alone: the
    first step is deterministic (same particles, same RNG streams), so its
    counts agree exactly; later steps diverge only through compaction order."""
    from cudapic_b200.batch import Batch
    specs = _small_specs(4)
    with Batch(specs) as b:
        b.run_steps(1)
        together = b.counts()
    alone = []
    for s in specs:
        with Batch([s]) as one:
            one.run_steps(1)
            alone.append(one.counts()[0])
    assert together == alone
