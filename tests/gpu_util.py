"""Helpers of the GPU tests: numpy <-> CUDA tensors (torch is only the
device-memory plumbing; every kernel call goes through libcudapic's C ABI)."""
import numpy as np


def dev(a):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    return torch.from_numpy(a.copy()).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    a = t.detach().cpu().numpy()
    return a.view(np.uint32) if a.dtype == np.int32 else a


def device_array(ptr, n, dtype):
    """Copies n elements at a device address (a library buffer) to the host;
    the caller has synchronised the stream that wrote them."""
    from cuda.bindings import runtime as rt
    out = np.empty(n, dtype)
    if n:
        err = rt.cudaMemcpy(out.ctypes.data, int(ptr), out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)[0]
        assert err == rt.cudaError_t.cudaSuccess, err
    return out


def counter(v):
    return dev(np.array([v], np.uint32))


def zeros(n, dtype=np.float32):
    return dev(np.zeros(n, dtype))


def rows(*cols):
    """Rows of float32/uint32 columns as one uint32 matrix (bit patterns)."""
    return np.stack([np.ascontiguousarray(c).view(np.uint32) for c in cols], axis=1)


def sorted_rows(*cols):
    r = rows(*cols)
    if r.shape[0] == 0:
        return r
    order = np.lexsort(r.T[::-1])
    return r[order]


def check_step_electrons(K, oracle, tables, dev_tables, g, ph, x, vx, vy, vz, ef, cap, seed=(3, 1, 4, 1), n_i0=1000):
    """Runs the fused electron step through the C ABI and checks it against
    the oracle's move_and_compact followed by its check_collisions_e over the
    survivors (with the fused step's algebraic scattering arithmetic), each
    survivor drawing from the RNG stream of its source slot.
    RNG planes (every slot), electron and ion sets bit-exact; densities within
    the deposit tolerance.  Returns (survivors, electrons after, ions after)."""
    cs, se, _ = tables
    dcs, dse, _ = dev_tables
    n = len(x)
    pad = lambda a, dt=np.float32: np.concatenate([a, np.zeros(cap - len(a), dt)])  # noqa: E731
    rng = [pad(np.asarray(p), np.uint32) for p in oracle.seed_streams(list(seed), cap)]
    rx, rvx, rvy, rvz, src = oracle.move_and_compact(ef, x, vx, vy, vz, g.factor_e, g.dt_e, ph)
    m = rx.size
    e_h = [pad(a) for a in (rx, rvx, rvy, rvz)]
    r_sub = [pad(p[src], np.uint32) for p in rng]
    i_h = [pad(np.full(n_i0, 0.0125, np.float32)) for _ in range(4)]
    _, ne_ref, ni_ref, dropped = oracle.check_collisions_e(se, cs, m, e_h, r_sub, i_h, m, n_i0, ph, algebraic=True)
    assert dropped == 0
    r_ref = [p.copy() for p in rng]
    for k in range(4):
        r_ref[k][src] = r_sub[k][:m]
    src_d = [dev(pad(a)) for a in (x, vx, vy, vz)]
    dst_d = [zeros(cap) for _ in range(4)]
    r_d = [dev(p) for p in rng]
    i_d = [dev(pad(np.full(n_i0, 0.0125, np.float32))) for _ in range(4)]
    alive, n_i = counter(0), counter(n_i0)
    de, di = zeros(len(ef)), zeros(len(ef))
    K.step_electrons(dev(ef), *src_d, *dst_d, *r_d, dse, dcs, float(se.max()), *i_d, alive, counter(n), n_i, de, di,
                     g)
    ne, ni = int(host(alive)[0]), int(host(n_i)[0])
    assert (ne, ni) == (ne_ref, ni_ref)
    for d, h in zip(r_d, r_ref):
        assert np.array_equal(host(d), h)
    got = [host(d)[:ne] for d in dst_d]
    assert np.array_equal(sorted_rows(*got), sorted_rows(*[h[:ne] for h in e_h]))
    gi = [host(d) for d in i_d]
    assert np.array_equal(sorted_rows(*[a[n_i0:ni] for a in gi]), sorted_rows(*[h[n_i0:ni] for h in i_h]))
    ref_e = oracle.get_density_f64(got[0], ph)
    assert np.linalg.norm(host(de) - ref_e) / np.linalg.norm(ref_e) < 2e-5
    if ni > n_i0:
        ref_i = oracle.get_density_f64(gi[0][n_i0:ni], ph)
        assert np.linalg.norm(host(di) - ref_i) / np.linalg.norm(ref_i) < 2e-5
    return m, ne, ni


def dead_mask(n, frac, seed=7):
    """Slots emptied by earlier in-place steps (x = CUDAPIC_DEAD_X)."""
    return np.random.default_rng(seed).random(n) < frac


def check_step_electrons_with_dead(K, oracle, tables, dev_tables, g, ph, x, vx, vy, vz, ef, cap, dead,
                                   seed=(3, 1, 4, 1), n_i0=1000):
    """The compacting fused step on planes with emptied slots: the oracle's
    move_and_compact + check_collisions_e over the live slots only (each
    survivor with its own slot's stream).  Electron and ion sets and every
    RNG plane bit-exact."""
    cs, se, _ = tables
    dcs, dse, _ = dev_tables
    n = len(x)
    x = np.where(dead, np.float32(-1.0), x).astype(np.float32)
    live = np.nonzero(~dead)[0]
    pad = lambda a, dt=np.float32: np.concatenate([a, np.zeros(cap - len(a), dt)])  # noqa: E731
    rng = [pad(np.asarray(p), np.uint32) for p in oracle.seed_streams(list(seed), cap)]
    rx, rvx, rvy, rvz, src = oracle.move_and_compact(ef, x[live], vx[live], vy[live], vz[live], g.factor_e, g.dt_e,
                                                     ph)
    m = rx.size
    slots = live[src]
    e_h = [pad(a) for a in (rx, rvx, rvy, rvz)]
    r_sub = [pad(p[slots], np.uint32) for p in rng]
    i_h = [pad(np.full(n_i0, 0.0125, np.float32)) for _ in range(4)]
    _, ne_ref, ni_ref, dropped = oracle.check_collisions_e(se, cs, m, e_h, r_sub, i_h, m, n_i0, ph, algebraic=True)
    assert dropped == 0
    r_ref = [p.copy() for p in rng]
    for k in range(4):
        r_ref[k][slots] = r_sub[k][:m]
    src_d = [dev(pad(a)) for a in (x, vx, vy, vz)]
    dst_d = [zeros(cap) for _ in range(4)]
    r_d = [dev(p) for p in rng]
    i_d = [dev(pad(np.full(n_i0, 0.0125, np.float32))) for _ in range(4)]
    alive, n_i = counter(0), counter(n_i0)
    de, di = zeros(len(ef)), zeros(len(ef))
    K.step_electrons(dev(ef), *src_d, *dst_d, *r_d, dse, dcs, float(se.max()), *i_d, alive, counter(n), n_i, de, di,
                     g)
    ne, ni = int(host(alive)[0]), int(host(n_i)[0])
    assert (ne, ni) == (ne_ref, ni_ref)
    for d, h in zip(r_d, r_ref):
        assert np.array_equal(host(d), h)
    got = [host(d)[:ne] for d in dst_d]
    assert np.all(got[0] >= 0.0)
    assert np.array_equal(sorted_rows(*got), sorted_rows(*[h[:ne] for h in e_h]))
    gi = [host(d) for d in i_d]
    assert np.array_equal(sorted_rows(*[a[n_i0:ni] for a in gi]), sorted_rows(*[h[n_i0:ni] for h in i_h]))
    ref_e = oracle.get_density_f64(got[0], ph)
    assert np.linalg.norm(host(de) - ref_e) / np.linalg.norm(ref_e) < 2e-5
    return m, ne, ni


def check_step_inplace(K, oracle, tables, dev_tables, g, ph, x, vx, vy, vz, ef, cap, dead, seed=(3, 1, 4, 1),
                       n_i0=1000, dens_tol=2e-5):
    """The in-place electron step (stream pass + scatter pass) through the C
    ABI against the oracle's move_and_compact + check_collisions_e over the
    live slots, every electron keeping its slot:
      * every slot [0, n): x, vx, vy, vz and the four RNG words bit-exact
        (absorbed electrons marked x = -1 with vx, vy, vz and RNG untouched,
        emptied slots untouched);
      * one collider record per collision event; spawned electrons at slots
        n, n + 1, ... and spawned ions: bit-exact as sets;
      * the next-step densities within the deposit tolerance of a fresh FP64
        deposit of the electrons (and spawned ions) present afterwards;
      * the collider count and the scatter ticket back at zero.
    Returns (survivors, electron slots after, ions after, colliders)."""
    cs, se, _ = tables
    dcs, dse, _ = dev_tables
    n = len(x)
    x = np.where(dead, np.float32(-1.0), x).astype(np.float32)
    live = np.nonzero(~dead)[0]
    pad = lambda a, dt=np.float32: np.concatenate([a, np.zeros(cap - len(a), dt)])  # noqa: E731
    rng = [pad(np.asarray(p), np.uint32) for p in oracle.seed_streams(list(seed), cap)]
    rx, rvx, rvy, rvz, src = oracle.move_and_compact(ef, x[live], vx[live], vy[live], vz[live], g.factor_e, g.dt_e,
                                                     ph)
    m = rx.size
    slots = live[src]
    e_h = [pad(a) for a in (rx, rvx, rvy, rvz)]
    r_sub = [pad(p[slots], np.uint32) for p in rng]
    i_h = [pad(np.full(n_i0, 0.0125, np.float32)) for _ in range(4)]
    events, ne_ref, ni_ref, dropped = oracle.check_collisions_e(se, cs, m, e_h, r_sub, i_h, m, n_i0, ph,
                                                                algebraic=True)
    assert dropped == 0
    exp = [pad(a).copy() for a in (x, vx, vy, vz)]
    exp[0][np.setdiff1d(live, slots)] = -1.0
    for k in range(4):
        exp[k][slots] = e_h[k][:m]
    r_ref = [p.copy() for p in rng]
    for k in range(4):
        r_ref[k][slots] = r_sub[k][:m]
    e_d = [dev(pad(a)) for a in (x, vx, vy, vz)]
    r_d = [dev(p) for p in rng]
    i_d = [dev(pad(np.full(n_i0, 0.0125, np.float32))) for _ in range(4)]
    n_e, n_i = counter(n), counter(n_i0)
    rec = [zeros(cap, np.uint32)] + [zeros(cap) for _ in range(3)] + [zeros(cap, np.uint32) for _ in range(4)]
    cnt, ticket = counter(0), counter(0)
    de, di = zeros(len(ef)), zeros(len(ef))
    K.step_electrons_inplace(dev(ef), *e_d, *r_d, dse, dcs, float(se.max()), n_e, rec, cnt, de, g)
    n_coll = int(host(cnt)[0])
    assert n_coll == int(np.count_nonzero(events))
    assert int(host(n_e)[0]) == n   # unchanged by the stream pass
    K.scatter_colliders_e(*e_d, *r_d, dcs, rec, cnt, ticket, *i_d, n_e, n_i, de, di, g)
    ne, ni = int(host(n_e)[0]), int(host(n_i)[0])
    assert (ne - n, ni) == (ne_ref - m, ni_ref)
    assert int(host(cnt)[0]) == 0 and int(host(ticket)[0]) == 0
    got = [host(d) for d in e_d]
    for k in range(4):
        assert np.array_equal(got[k][:n].view(np.uint32), exp[k][:n].view(np.uint32)), k
    for d, h in zip(r_d, r_ref):
        assert np.array_equal(host(d), h)
    gs, es = sorted_rows(*[a[n:ne] for a in got]), sorted_rows(*[h[m:ne_ref] for h in e_h])
    assert np.array_equal(gs, es), _row_diff(gs, es)
    gi = [host(d) for d in i_d]
    assert np.array_equal(sorted_rows(*[a[n_i0:ni] for a in gi]), sorted_rows(*[h[n_i0:ni] for h in i_h]))
    present = got[0][:ne][got[0][:ne] >= 0.0]
    ref_e = oracle.get_density_f64(present, ph)
    assert np.linalg.norm(host(de) - ref_e) / np.linalg.norm(ref_e) < dens_tol
    if ni > n_i0:
        ref_i = oracle.get_density_f64(gi[0][n_i0:ni], ph)
        assert np.linalg.norm(host(di) - ref_i) / np.linalg.norm(ref_i) < dens_tol
    return m, ne, ni, int(np.count_nonzero(events))


def _row_diff(got, exp):
    """Which columns differ between two sorted row sets, and a few rows."""
    if got.shape != exp.shape:
        return "shapes %s vs %s" % (got.shape, exp.shape)
    bad = np.nonzero(np.any(got != exp, axis=1))[0]
    cols = np.any(got != exp, axis=0)
    return "%d of %d rows differ, columns %s; first: got %s exp %s" % (
        len(bad), len(got), np.nonzero(cols)[0].tolist(), got[bad[:3]].view(np.float32).tolist(),
        exp[bad[:3]].view(np.float32).tolist())
