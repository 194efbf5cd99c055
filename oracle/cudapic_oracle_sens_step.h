/*
 * cudapic_oracle_sens_step.h -- one forward step of the slot-form model of
 * the voltage-sensitivity path, in the arithmetic the including file selects:
 *
 *   SENS_F32 1   the f32 arithmetic of the CUDA path (2^-20 fixed-point
 *                deposit, FP64 Poisson sums with f32 output, f32 push and
 *                algebraic scattering, the oracle's deterministic
 *                transcendentals), bit-exact against it;
 *   SENS_F32 0   the same model in double (exact CIC weights, libm).
 *
 * Included twice by cudapic_oracle_sens.c.  TEST INFRASTRUCTURE ONLY.
 *
 * Slot form of the reference step (Rust-CUDA/src/main.rs:1725-1808): the
 * same kernels in the same order -- densities, Poisson, electron push, ion
 * push (every N_SUB-th step), electron collisions with their spawns, ion
 * collisions -- but particles keep their slots: an absorbed particle is
 * marked dead (x = -1) instead of being compacted away, and the spawns of a
 * step take the next free slots in the slot order of their parents.  Every
 * particle keeps one RNG stream for its whole life, so the run is a
 * deterministic function of the initial state and the voltage.
 */
#if SENS_F32
#define R float
#define FN(name) name##_f32
#define SQRT sqrtf
#define FABS fabsf
#define TAN orc_tanf
#define ATAN orc_atanf
#define SIN orc_sinf
#define COS orc_cosf
#define RK(c) c##f
#else
#define R double
#define FN(name) name##_f64
#define SQRT sqrt
#define FABS fabs
#define TAN tan
#define ATAN atan
#define SIN sin
#define COS cos
#define RK(c) c
#endif

typedef struct FN(sp) {
    R *x, *vx, *vy, *vz;
    uint32_t *r[4];
    uint32_t n, cap;
} FN(sp);

/* get_density (Rust-CUDA/src/main.rs:356-406) over the live slots. */
static void FN(deposit)(const FN(sp) *s, const orc_phys *ph, R *dens) {
    const uint32_t n_g = ph->n_g;
#if SENS_F32
    uint64_t *acc = (uint64_t *)calloc(n_g, sizeof(uint64_t));
    for (uint32_t p = 0; p < s->n; ++p) {
        if (!(s->x[p] >= 0.0f)) continue;
        const float pos = s->x[p] * ph->inv_dx;
        const int c = cell_of(pos, n_g);
        const float rem = pos - (float)c;
        uint32_t r = (uint32_t)nearbyintf(rem * (float)(1u << SENS_DEP_Q));
        if (r > (1u << SENS_DEP_Q)) r = 1u << SENS_DEP_Q;
        acc[c] += (1u << SENS_DEP_Q) - r;
        acc[c + 1] += r;
    }
    const double w = ph->weight_factor_d * (1.0 / (double)(1u << SENS_DEP_Q));
    for (uint32_t k = 0; k < n_g; ++k) {
        float f = (float)((double)acc[k] * w);
        if (k == 0 || k == n_g - 1) f *= 2.0f;
        dens[k] = f;
    }
    free(acc);
#else
    const double inv_dx = 1.0 / ph->dx;
    for (uint32_t k = 0; k < n_g; ++k) dens[k] = 0.0;
    for (uint32_t p = 0; p < s->n; ++p) {
        if (!(s->x[p] >= 0.0)) continue;
        const double pos = s->x[p] * inv_dx;
        int c = (int)pos;
        if (c > (int)n_g - 2) c = (int)n_g - 2;
        if (c < 0) c = 0;
        const double rem = pos - c;
        dens[c] += (1.0 - rem) * ph->weight_factor_d;
        dens[c + 1] += rem * ph->weight_factor_d;
    }
    dens[0] *= 2.0;
    dens[n_g - 1] *= 2.0;
#endif
}

/* solve_poisson_scan_f32 (Rust-CUDA/src/main.rs:408-494) with FP64 sums:
 * the closed form of the CUDA solve (two prefix sums), f32 or double output. */
static void FN(poisson)(const R *ne, const R *ni, R pot0, const orc_phys *ph, R *efield) {
    const int n = (int)ph->n_g;
    const double e_charge = 1.60217662e-19;
    const double alpha = -ph->dx * ph->dx / 8.85418781e-12;
    double *rho = (double *)malloc(sizeof(double) * n);
    double *G = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n);
    double *Rs = (double *)malloc(sizeof(double) * n);
    double *pot = (double *)malloc(sizeof(double) * n);
    const double p0 = (double)pot0;
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
        rho[i] = e_charge * ((double)ni[i] - (double)ne[i]);
        double gi = 0.0;
        if (i != 0) gi = (double)i * (alpha * rho[i] - (i == 1 ? p0 : 0.0));
        acc += gi;
        G[i] = acc;
    }
    acc = 0.0;
    for (int i = 0; i < n; ++i) {
        double ri = 0.0;
        if (i != 0 && i < n - 1) ri = (-G[i] / ((double)i + 1.0)) / (double)i;
        r[i] = ri;
        acc += ri;
        Rs[i] = acc;
    }
    const double r_total = Rs[n - 2];
    for (int i = 0; i < n; ++i) {
        if (i == 0) pot[i] = p0;
        else if (i < n - 1) pot[i] = (double)i * (r_total - Rs[i] + r[i]);
        else pot[i] = 0.0;
    }
    const double inv_dx = 1.0 / ph->dx, half_inv_dx = 0.5 / ph->dx;
    const double hdx_eps = ph->dx / (2.0 * 8.85418781e-12);
    for (int i = 0; i < n; ++i) {
        double e;
        if (i == 0) e = (pot[0] - pot[1]) * inv_dx - rho[0] * hdx_eps;
        else if (i == n - 1) e = (pot[n - 2] - pot[n - 1]) * inv_dx + rho[n - 1] * hdx_eps;
        else e = (pot[i - 1] - pot[i + 1]) * half_inv_dx;
        efield[i] = (R)e;
    }
    free(rho); free(G); free(r); free(Rs); free(pot);
}

/* move_and_compact's push (Rust-CUDA/src/main.rs:596-620) of the live slots
 * in place; a particle leaving [0, L] is marked dead.  obs (may be null)
 * receives the observable sum of the species: electrons the <j E> term
 * (v + 1/2 f E(x)) E(x), ions the flux term v c2 of the cell at the grounded
 * electrode.  tape (may be null): x and v before the push. */
static void FN(push)(FN(sp) *s, const R *E, R f, R dt, R gap, const orc_phys *ph, int ions, double *obs,
                     double *tape_x, double *tape_v) {
    const uint32_t n_g = ph->n_g;
#if SENS_F32
    const float inv_dx = ph->inv_dx;
#else
    const double inv_dx = 1.0 / ph->dx;
#endif
    for (uint32_t p = 0; p < s->n; ++p) {
        const R x = s->x[p], vx = s->vx[p];
        if (tape_x) {
            tape_x[p] = (double)x;
            tape_v[p] = (double)vx;
        }
        if (!(x >= (R)0)) continue;
        const R pos = x * inv_dx;
#if SENS_F32
        const int c = cell_of(pos, n_g);
#else
        int c = (int)pos;
        if (c > (int)n_g - 2) c = (int)n_g - 2;
        if (c < 0) c = 0;
#endif
        const R c2 = pos - (R)c;
        const R ex = ((R)1 - c2) * E[c] + c2 * E[c + 1];
        if (obs) {
            if (!ions) *obs += ((double)vx + 0.5 * (double)f * (double)ex) * (double)ex;
            else if (c == (int)n_g - 2) *obs += (double)vx * (double)c2;
        }
        const R v1 = vx + f * ex;
        const R x1 = x + v1 * dt;
        s->vx[p] = v1;
        s->x[p] = (x1 >= (R)0 && x1 <= gap) ? x1 : (R)-1;
    }
}

typedef struct FN(consts) {
    R f1, f2, me, qe, exc_j, ion_j, hme, hmu, nr, dt_e, dt_i;
} FN(consts);

static void FN(consts_init)(FN(consts) *k, const orc_phys *ph) {
    k->f1 = (R)ph->f1;
    k->f2 = (R)ph->f2;
    k->me = (R)(float)ORC_E_MASS;
    k->qe = (R)(float)ORC_E_CHARGE;
    k->exc_j = RK(11.5) * k->qe;
    k->ion_j = RK(15.8) * k->qe;
    k->hme = (R)ph->half_me_over_e;
    k->hmu = (R)ph->half_mu_over_e;
    k->nr = (R)ph->normal_range;
    k->dt_e = (R)ph->dt_e;
    k->dt_i = (R)ph->dt_i;
}

static inline void FN(euler_alg)(R gx, R gy, R gz, R *st, R *ct, R *sp, R *cp) {
    const R r2 = gy * gy + gz * gz;
    const R r = SQRT(r2);
    if (gx == (R)0) {
        *st = (R)1;
        *ct = (R)0;
    } else {
        const R gn = SQRT(gx * gx + r2);
        *st = r / gn;
        *ct = gx / gn;
    }
    if (gy == (R)0) {
        *sp = (gz > (R)0) ? (R)1 : (R)-1;
        *cp = (R)0;
    } else {
        *sp = gz / r;
        *cp = gy / r;
    }
}

static inline void FN(sincos_acos)(R c, R *s, R *co) {
    R t = ((R)1 - c) * ((R)1 + c);
    *s = SQRT(t > (R)0 ? t : (R)0);
    *co = c;
}

static inline void FN(rot)(R g, R sc, R cc, R se, R ce, R st, R ct, R sp, R cp, R *ox, R *oy, R *oz) {
    *ox = g * (ct * cc - st * sc * ce);
    *oy = g * (st * cp * cc + ct * cp * sc * ce - sp * sc * se);
    *oz = g * (st * sp * cc + ct * sp * sc * ce + cp * sc * se);
}

/* collision_e (Rust-CUDA/src/main.rs:1035-1165) with the algebraic sines
 * and cosines, draws given: ev 1 elastic / 2 excitation (a = cos chi draw
 * 1 - 2u), ev 3 ionization (a = the energy-sharing draw u); eta = 2 pi u.
 * out: the scattered velocity; child (ev 3): the new electron. */
static void FN(scatter_e)(const FN(consts) *k, const R v[3], int ev, R a, R eta, R out[3], R child[3]) {
    const R gx = v[0], gy = v[1], gz = v[2];
    R gm = SQRT(gx * gx + gy * gy + gz * gz);
    const R wx = k->f1 * gx, wy = k->f1 * gy, wz = k->f1 * gz;
    R st, ct, sp, cp;
    FN(euler_alg)(gx, gy, gz, &st, &ct, &sp, &cp);
    R chi_s, chi_c, se, ce;
    if (ev == 1) {
        FN(sincos_acos)(a, &chi_s, &chi_c);
    } else if (ev == 2) {
        R en = RK(0.5) * k->me * gm * gm;
        en = FABS(en - k->exc_j);
        gm = SQRT(RK(2.0) * en / k->me);
        FN(sincos_acos)(a, &chi_s, &chi_c);
    } else {
        R en = RK(0.5) * k->me * gm * gm;
        en = FABS(en - k->ion_j);
        const R e_new = RK(10.0) * TAN(a * ATAN(en / k->qe / RK(20.0))) * k->qe;
        const R e_orig = FABS(en - e_new);
        gm = SQRT(RK(2.0) * e_orig / k->me);
        const R g_new = SQRT(RK(2.0) * e_new / k->me);
        R sc2, cc2, nx, ny, nz;
        FN(sincos_acos)(SQRT(e_new / en), &sc2, &cc2);
        se = SIN(eta);
        ce = COS(eta);
        FN(rot)(g_new, sc2, cc2, -se, -ce, st, ct, sp, cp, &nx, &ny, &nz);
        child[0] = wx + k->f2 * nx;
        child[1] = wy + k->f2 * ny;
        child[2] = wz + k->f2 * nz;
        FN(sincos_acos)(SQRT(e_orig / en), &chi_s, &chi_c);
    }
    if (ev != 3) {
        se = SIN(eta);
        ce = COS(eta);
    }
    R nx, ny, nz;
    FN(rot)(gm, chi_s, chi_c, se, ce, st, ct, sp, cp, &nx, &ny, &nz);
    out[0] = wx + k->f2 * nx;
    out[1] = wy + k->f2 * ny;
    out[2] = wz + k->f2 * nz;
}

/* collision_i (Rust-CUDA/src/main.rs:1221-1292) with the algebraic sines and
 * cosines: ev 4 isotropic (c = 1 - 2u), ev 5 backscatter (chi = pi, exactly). */
static void FN(scatter_i)(const R v[3], const R t[3], int ev, R c, R eta, R out[3]) {
    const R gx = v[0] - t[0], gy = v[1] - t[1], gz = v[2] - t[2];
    const R gg = SQRT(gx * gx + gy * gy + gz * gz);
    const R wx = RK(0.5) * (v[0] + t[0]), wy = RK(0.5) * (v[1] + t[1]), wz = RK(0.5) * (v[2] + t[2]);
    R st, ct, sp, cp, sc, cc;
    FN(euler_alg)(gx, gy, gz, &st, &ct, &sp, &cp);
    if (ev == 4) {
        FN(sincos_acos)(c, &sc, &cc);
    } else {
        sc = (R)0;
        cc = (R)-1;
    }
    const R se = SIN(eta), ce = COS(eta);
    R nx, ny, nz;
    FN(rot)(gg, sc, cc, se, ce, st, ct, sp, cp, &nx, &ny, &nz);
    out[0] = wx + RK(0.5) * nx;
    out[1] = wy + RK(0.5) * ny;
    out[2] = wz + RK(0.5) * nz;
}

static inline R FN(draw)(rng4 *r) { return (R)draw(r); }

/* check_collisions_e (Rust-CUDA/src/main.rs:971-1033) over the slots live
 * before the step's spawns, then the spawns in parent slot order. */
static void FN(collide_e)(FN(sp) *e, FN(sp) *ion, const float *sig_e, const float *cs, const FN(consts) *k,
                          tape_step *ts, uint32_t *dev_err) {
    const uint32_t n0 = e->n, ni0 = ion->n;
    uint32_t spawned = 0;
    for (uint32_t p = 0; p < n0; ++p) {
        if (!(e->x[p] >= (R)0)) continue;
        rng4 rs = {{e->r[0][p], e->r[1][p], e->r[2][p], e->r[3][p]}};
        const R v[3] = {e->vx[p], e->vy[p], e->vz[p]};
        const R v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
#if SENS_F32
        const uint32_t idx = energy_index(k->hme * v2);
        const float a = sig_e[idx] * sqrtf(v2) * k->dt_e;
        const float u = draw(&rs);
        const int hit = (u >= a + 5e-7f) ? 0 : (u < 1.0f - orc_expf(-a));
#else
        double et = k->hme * v2 / 0.001 + 0.5;
        if (et > (double)(ORC_CS_RANGES - 1)) et = (double)(ORC_CS_RANGES - 1);
        const uint32_t idx = (uint32_t)et;
        const double a = (double)sig_e[idx] * sqrt(v2) * k->dt_e;
        const double u = (double)draw(&rs);
        const int hit = u < 1.0 - exp(-a);
#endif
        if (hit) {
            const R t0 = (R)cs[idx];
            const R t1 = t0 + (R)cs[ORC_CS_RANGES + idx];
            const R t2 = t1 + (R)cs[2 * ORC_CS_RANGES + idx];
            const R rnd = FN(draw)(&rs);
            int ev;
            R aa, eta;
            if (rnd < t0 / t2) {
                ev = 1;
                aa = RK(1.0) - RK(2.0) * FN(draw)(&rs);
                eta = (R)F_TWO_PI * FN(draw)(&rs);
            } else if (rnd < t1 / t2) {
                ev = 2;
                aa = RK(1.0) - RK(2.0) * FN(draw)(&rs);
                eta = (R)F_TWO_PI * FN(draw)(&rs);
            } else {
                ev = 3;
                aa = FN(draw)(&rs);
                eta = (R)F_TWO_PI * FN(draw)(&rs);
            }
            R out[3], child[3];
            FN(scatter_e)(k, v, ev, aa, eta, out, child);
            uint32_t ce = SENS_NO_SLOT, ci = SENS_NO_SLOT;
            if (ev == 3) {
                float ta, tb, tc;
                three_normal(&rs, ph_normal_range_f(k), &ta, &tb, &tc);
                const uint32_t se_ = n0 + spawned, si_ = ni0 + spawned;
                ++spawned;
                if (se_ < e->cap) {
                    e->x[se_] = e->x[p];
                    e->vx[se_] = child[0];
                    e->vy[se_] = child[1];
                    e->vz[se_] = child[2];
                    ce = se_;
                } else {
                    *dev_err |= 0x1u;
                }
                if (si_ < ion->cap) {
                    ion->x[si_] = e->x[p];
                    ion->vx[si_] = (R)ta;
                    ion->vy[si_] = (R)tb;
                    ion->vz[si_] = (R)tc;
                    ci = si_;
                } else {
                    *dev_err |= 0x2u;
                }
            }
            e->vx[p] = out[0];
            e->vy[p] = out[1];
            e->vz[p] = out[2];
            if (ts) {
                rec_e rr = {p, (uint32_t)ev, ce, ci, {(double)v[0], (double)v[1], (double)v[2]}, (double)aa,
                            (double)eta};
                tape_push_e(ts, &rr);
            }
        }
        e->r[0][p] = rs.s[0]; e->r[1][p] = rs.s[1]; e->r[2][p] = rs.s[2]; e->r[3][p] = rs.s[3];
    }
    e->n = n0 + spawned < e->cap ? n0 + spawned : e->cap;
    ion->n = ni0 + spawned < ion->cap ? ni0 + spawned : ion->cap;
}

/* check_collisions_i (Rust-CUDA/src/main.rs:1167-1219) over the live ions,
 * the step's spawns included. */
static void FN(collide_i)(FN(sp) *ion, const float *sig_i, const float *cs, const FN(consts) *k, tape_step *ts) {
    for (uint32_t p = 0; p < ion->n; ++p) {
        if (!(ion->x[p] >= (R)0)) continue;
        rng4 rs = {{ion->r[0][p], ion->r[1][p], ion->r[2][p], ion->r[3][p]}};
        float ta, tb, tc;
        three_normal(&rs, ph_normal_range_f(k), &ta, &tb, &tc);
        const R t[3] = {(R)ta, (R)tb, (R)tc};
        const R v[3] = {ion->vx[p], ion->vy[p], ion->vz[p]};
        const R gx = v[0] - t[0], gy = v[1] - t[1], gz = v[2] - t[2];
        const R g2 = gx * gx + gy * gy + gz * gz;
#if SENS_F32
        const uint32_t idx = energy_index(k->hmu * g2);
        const float a = sig_i[idx] * sqrtf(g2) * k->dt_i;
        const float u = draw(&rs);
        const int hit = (u >= a + 5e-7f) ? 0 : (u < 1.0f - orc_expf(-a));
#else
        double et = k->hmu * g2 / 0.001 + 0.5;
        if (et > (double)(ORC_CS_RANGES - 1)) et = (double)(ORC_CS_RANGES - 1);
        const uint32_t idx = (uint32_t)et;
        const double a = (double)sig_i[idx] * sqrt(g2) * k->dt_i;
        const double u = (double)draw(&rs);
        const int hit = u < 1.0 - exp(-a);
#endif
        if (hit) {
            const R t0 = (R)cs[3 * ORC_CS_RANGES + idx];
            const R t1 = t0 + (R)cs[4 * ORC_CS_RANGES + idx];
            const R rnd = FN(draw)(&rs);
            int ev;
            R c = RK(0.0);
            if (rnd < t0 / t1) {
                ev = 4;
                c = RK(1.0) - RK(2.0) * FN(draw)(&rs);
            } else {
                ev = 5;
            }
            const R eta = (R)F_TWO_PI * FN(draw)(&rs);
            R out[3];
            FN(scatter_i)(v, t, ev, c, eta, out);
            ion->vx[p] = out[0];
            ion->vy[p] = out[1];
            ion->vz[p] = out[2];
            if (ts) {
                rec_i rr = {p, (uint32_t)ev, {(double)v[0], (double)v[1], (double)v[2]},
                            {(double)t[0], (double)t[1], (double)t[2]}, (double)c, (double)eta};
                tape_push_i(ts, &rr);
            }
        }
        ion->r[0][p] = rs.s[0]; ion->r[1][p] = rs.s[1]; ion->r[2][p] = rs.s[2]; ion->r[3][p] = rs.s[3];
    }
}

/* One step t of the model.  obs[2] += (<j E> sum, ion flux sum); ts (may be
 * null) records what the adjoint needs. */
static void FN(step)(FN(sp) *e, FN(sp) *ion, R *dens_e, R *dens_i, R *E, const orc_phys *ph, const float *sig_e,
                     const float *sig_i, const float *cs, double voltage, uint64_t t, double obs[2],
                     tape_step *ts, uint32_t *dev_err) {
    FN(consts) k;
    FN(consts_init)(&k, ph);
    const int ion_step = (t % ph->n_sub) == 0;
    const double cosv = cos(((double)(t % ph->n_t) / (double)ph->n_t) * (2.0 * 3.141592653589793));
#if SENS_F32
    const float pot0 = (float)(voltage * cos(((double)(t % ph->n_t) / (double)ph->n_t) * (2.0 * 3.141592653589793)));
    const float gap = ph->gap;
#else
    const double pot0 = voltage * cosv;
    const double gap = (double)ph->gap;
#endif
    FN(deposit)(e, ph, dens_e);
    if (ion_step) FN(deposit)(ion, ph, dens_i);
    FN(poisson)(dens_e, dens_i, pot0, ph, E);
    if (ts) {
        tape_begin(ts, e->n, ion_step ? ion->n : 0, ph->n_g, ion_step, cosv);
        for (uint32_t j = 0; j < ph->n_g; ++j) ts->E[j] = (double)E[j];
    }
    FN(push)(e, E, (R)ph->factor_e, (R)ph->dt_e, gap, ph, 0, &obs[0], ts ? ts->xe : NULL, ts ? ts->vxe : NULL);
    if (ion_step)
        FN(push)(ion, E, (R)ph->factor_i, (R)ph->dt_i, gap, ph, 1, &obs[1], ts ? ts->xi : NULL, ts ? ts->vxi : NULL);
    FN(collide_e)(e, ion, sig_e, cs, &k, ts, dev_err);
    if (ion_step) FN(collide_i)(ion, sig_i, cs, &k, ts);
}

#undef R
#undef FN
#undef SQRT
#undef FABS
#undef TAN
#undef ATAN
#undef SIN
#undef COS
#undef RK
