"""GPU test of cudapic_step_electrons_noalloc: the fused electron step for
callers that cannot allocate device memory (their device memory belongs to
a host pool or framework that hands this library only its particle
buffers), so the kernel's slot counter and completion ticket live in a
static device array of the library and the new count is written into n_e.

Two calls in a row, each against cudapic_step_electrons on the same inputs:
the second call runs on the static array as the first one left it (the
kernel's last CTA resets both counters itself, and the entry point also
clears them on the stream before every launch).  The file name makes
pytest collect it last, so a run that stops at the first failure has run
every other test before it."""
import numpy as np
import pytest

from gpu_util import counter, dev, host, sorted_rows, zeros

pytestmark = pytest.mark.gpu

E_MASS = 9.10938356e-31


def _run(K, fn, g, ef, tabs, src, rng, n_e, ions, n_i, cap):
    """One fused electron step on fresh device copies of the inputs; returns
    host copies of every output."""
    dcs, dse, smax = tabs
    src_d = [dev(a) for a in src]
    dst_d = [zeros(cap) for _ in range(4)]
    rng_d = [dev(p) for p in rng]
    ion_d = [dev(a) for a in ions]
    ne_d, ni_d = counter(n_e), counter(n_i)
    de, di = zeros(400), zeros(400)
    if fn == "noalloc":
        K.step_electrons_noalloc(ef, *src_d, *dst_d, *rng_d, dse, dcs, smax, *ion_d, ne_d, ni_d, de, di, g)
        ne = int(host(ne_d)[0])
    else:
        alive = counter(0)
        K.step_electrons(ef, *src_d, *dst_d, *rng_d, dse, dcs, smax, *ion_d, alive, ne_d, ni_d, de, di, g)
        ne = int(host(alive)[0])
        assert int(host(ne_d)[0]) == n_e   # the existing entry leaves the input count alone
    ni = int(host(ni_d)[0])
    return dict(ne=ne, ni=ni, dst=[host(d) for d in dst_d], rng=[host(p) for p in rng_d],
                ions=[host(a) for a in ion_d], de=host(de).astype(np.float64), di=host(di).astype(np.float64))


def test_noalloc_step_matches_step_electrons_on_two_calls(cudapic, tables, cuda_device):
    from cudapic_b200.workloads import field_profile, steady_state
    K = cudapic.kernels
    cs, se, _ = tables
    tabs = (dev(cs), dev(se), float(se.max()))
    n, n_i0 = 300_001, 1000
    cap = (2 * n + 4096 + 3) // 4 * 4
    g = cudapic.grid_from_params(n_t=100, capacity=cap)   # long steps: many collisions and ionizations
    ef = dev(field_profile(400))
    pad = lambda a, dt=np.float32: np.concatenate([a, np.zeros(cap - len(a), dt)])  # noqa: E731
    src = [pad(a) for a in steady_state(n, E_MASS, 60.0, dt=g.dt_e, seed=5)]
    planes = [zeros(cap, np.uint32) for _ in range(4)]
    K.xoshiro128_seed_streams([7, 7, 1, 3], cap, *planes)
    rng = [host(p) for p in planes]
    ions = [pad(np.full(n_i0, 0.0125, np.float32)) for _ in range(4)]
    n_e, n_i = n, n_i0
    for call in range(2):
        a = _run(K, "existing", g, ef, tabs, src, rng, n_e, ions, n_i, cap)
        b = _run(K, "noalloc", g, ef, tabs, src, rng, n_e, ions, n_i, cap)
        assert (b["ne"], b["ni"]) == (a["ne"], a["ni"]), call
        assert a["ne"] != n_e and a["ni"] > n_i       # absorption and ionization happened
        for pa, pb in zip(a["rng"], b["rng"]):
            assert np.array_equal(pa, pb)
        ne, ni = a["ne"], a["ni"]
        assert np.array_equal(sorted_rows(*[d[:ne] for d in b["dst"]]), sorted_rows(*[d[:ne] for d in a["dst"]]))
        assert np.array_equal(sorted_rows(*[d[n_i:ni] for d in b["ions"]]),
                              sorted_rows(*[d[n_i:ni] for d in a["ions"]]))
        for key in ("de", "di"):   # f32 atomic sums in another order: the deposit tolerance
            assert np.linalg.norm(b[key] - a[key]) / np.linalg.norm(a[key]) < 2e-5, (call, key)
        # the next call starts from this call's results
        src, rng, ions, n_e, n_i = b["dst"], b["rng"], b["ions"], ne, ni
