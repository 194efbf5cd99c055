/*
 * cudapic_oracle_sens.c -- CPU restatement of the voltage-sensitivity path:
 * the slot-form model of the PIC/MCC step (cudapic_oracle_sens_step.h) and
 * its pathwise adjoint with collision events and random draws frozen.
 *
 * TEST INFRASTRUCTURE ONLY (see cudapic_oracle.h): the checker of the CUDA
 * sensitivity kernels, never part of the product path.
 *
 * Observables (time averages over the window of K steps):
 *   J_P  electron power absorption <j E> averaged over the gap [W m^-3]:
 *        -e (W/A) / L / K * sum_steps sum_electrons (v + f E(x)/2) E(x), the
 *        time-centred velocity of the push times the field at the particle
 *        (eduPIC's <j E>, C/eduPIC.cc:593-614, :1011-1026, per particle);
 *   J_G  ion flux to the grounded electrode [m^-2 s^-1]: the CIC flux
 *        density n v at node N_G-1 (boundary node doubled, as the density),
 *        2 (W/A)/dx / K_i * sum_ion_steps sum_ions v c2 [cell N_G-2], a smooth
 *        estimate of the counted flux of C/eduPIC.cc:651-658.
 *
 * The adjoint runs in double on the recorded trajectory: collision
 * Jacobians by central differences of the double scattering, the Poisson
 * adjoint by a Thomas solve (the CUDA path uses the scan form), push and
 * deposit adjoints in closed form.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cudapic_oracle.h"
#include "cudapic_oracle_mcc.h"

#define SENS_DEP_Q 20
#define SENS_NO_SLOT 0xFFFFFFFFu

typedef struct rec_e {
    uint32_t p, ev, ce, ci;
    double v[3];
    double a, eta;
} rec_e;

typedef struct rec_i {
    uint32_t p, ev;
    double v[3], t[3];
    double c, eta;
} rec_i;

typedef struct tape_step {
    uint32_t ne, ni;
    int ion;
    double cosv;
    double *xe, *vxe, *xi, *vxi, *E;
    rec_e *re;
    uint32_t nre, cre;
    rec_i *ri;
    uint32_t nri, cri;
} tape_step;

static void tape_begin(tape_step *ts, uint32_t ne, uint32_t ni, uint32_t n_g, int ion, double cosv) {
    ts->ne = ne;
    ts->ni = ni;
    ts->ion = ion;
    ts->cosv = cosv;
    ts->xe = (double *)malloc(sizeof(double) * (ne ? ne : 1));
    ts->vxe = (double *)malloc(sizeof(double) * (ne ? ne : 1));
    ts->xi = (double *)malloc(sizeof(double) * (ni ? ni : 1));
    ts->vxi = (double *)malloc(sizeof(double) * (ni ? ni : 1));
    ts->E = (double *)malloc(sizeof(double) * n_g);
}

static void tape_push_e(tape_step *ts, const rec_e *r) {
    if (ts->nre == ts->cre) {
        ts->cre = ts->cre ? 2 * ts->cre : 64;
        ts->re = (rec_e *)realloc(ts->re, sizeof(rec_e) * ts->cre);
    }
    ts->re[ts->nre++] = *r;
}

static void tape_push_i(tape_step *ts, const rec_i *r) {
    if (ts->nri == ts->cri) {
        ts->cri = ts->cri ? 2 * ts->cri : 64;
        ts->ri = (rec_i *)realloc(ts->ri, sizeof(rec_i) * ts->cri);
    }
    ts->ri[ts->nri++] = *r;
}

static void tape_free(tape_step *ts) {
    free(ts->xe); free(ts->vxe); free(ts->xi); free(ts->vxi); free(ts->E); free(ts->re); free(ts->ri);
}

#define ph_normal_range_f(k) ((float)(k)->nr)

#define SENS_F32 1
#include "cudapic_oracle_sens_step.h"
#undef SENS_F32
#define SENS_F32 0
#include "cudapic_oracle_sens_step.h"
#undef SENS_F32

/* ------------------------------------------------------------------ */
/* adjoint                                                             */
/* ------------------------------------------------------------------ */

/* d out / d v (row = output component) of the double scattering at the
 * recorded draws, by central differences. */
static void jac_e(const consts_f64 *k, const rec_e *r, double J[3][3], double Jc[3][3]) {
    double vm = sqrt(r->v[0] * r->v[0] + r->v[1] * r->v[1] + r->v[2] * r->v[2]);
    double h = 1e-6 * (vm > 1.0 ? vm : 1.0);
    for (int c = 0; c < 3; ++c) {
        double vp[3] = {r->v[0], r->v[1], r->v[2]}, vn[3] = {r->v[0], r->v[1], r->v[2]};
        vp[c] += h;
        vn[c] -= h;
        double op[3], on[3], cp[3] = {0, 0, 0}, cn[3] = {0, 0, 0};
        scatter_e_f64(k, vp, (int)r->ev, r->a, r->eta, op, cp);
        scatter_e_f64(k, vn, (int)r->ev, r->a, r->eta, on, cn);
        for (int o = 0; o < 3; ++o) {
            J[o][c] = (op[o] - on[o]) / (2.0 * h);
            Jc[o][c] = (cp[o] - cn[o]) / (2.0 * h);
        }
    }
}

static void jac_i(const rec_i *r, double J[3][3]) {
    double vm = sqrt(r->v[0] * r->v[0] + r->v[1] * r->v[1] + r->v[2] * r->v[2]);
    double h = 1e-6 * (vm > 1.0 ? vm : 1.0);
    for (int c = 0; c < 3; ++c) {
        double vp[3] = {r->v[0], r->v[1], r->v[2]}, vn[3] = {r->v[0], r->v[1], r->v[2]};
        vp[c] += h;
        vn[c] -= h;
        double op[3], on[3];
        scatter_i_f64(vp, r->t, (int)r->ev, r->c, r->eta, op);
        scatter_i_f64(vn, r->t, (int)r->ev, r->c, r->eta, on);
        for (int o = 0; o < 3; ++o) J[o][c] = (op[o] - on[o]) / (2.0 * h);
    }
}

/* Adjoint of the Poisson solve and field: eb (field adjoint) -> adjoints of
 * the electron and ion densities; returns the adjoint of pot0. */
static double poisson_adjoint(const double *eb, const orc_phys *ph, double *neb, double *nib) {
    const int n = (int)ph->n_g;
    const double e_charge = 1.60217662e-19;
    const double alpha = -ph->dx * ph->dx / 8.85418781e-12;
    const double inv_dx = 1.0 / ph->dx, half_inv_dx = 0.5 / ph->dx;
    const double hdx_eps = ph->dx / (2.0 * 8.85418781e-12);
    double *pb = (double *)calloc(n, sizeof(double));
    double *rb = (double *)calloc(n, sizeof(double));
    double *w = (double *)calloc(n, sizeof(double));
    double *g = (double *)calloc(n, sizeof(double));
    double *lam = (double *)calloc(n, sizeof(double));
    for (int i = 0; i < n; ++i) {
        if (i == 0) {
            pb[0] += eb[0] * inv_dx;
            pb[1] -= eb[0] * inv_dx;
            rb[0] -= eb[0] * hdx_eps;
        } else if (i == n - 1) {
            pb[n - 2] += eb[i] * inv_dx;
            rb[n - 1] += eb[i] * hdx_eps;
        } else {
            pb[i - 1] += eb[i] * half_inv_dx;
            pb[i + 1] -= eb[i] * half_inv_dx;
        }
    }
    /* T lam = pb on the interior nodes 1..n-2, T = tridiag(1, -2, 1) (symmetric) */
    w[1] = 1.0 / -2.0;
    g[1] = pb[1] / -2.0;
    for (int i = 2; i <= n - 2; ++i) {
        w[i] = 1.0 / (-2.0 - w[i - 1]);
        g[i] = (pb[i] - g[i - 1]) / (-2.0 - w[i - 1]);
    }
    lam[n - 2] = g[n - 2];
    for (int i = n - 3; i >= 1; --i) lam[i] = g[i] - w[i] * lam[i + 1];
    for (int i = 1; i <= n - 2; ++i) rb[i] += alpha * lam[i];
    const double pot0b = pb[0] - lam[1];
    for (int i = 0; i < n; ++i) {
        neb[i] = -e_charge * rb[i];
        nib[i] = e_charge * rb[i];
    }
    free(pb); free(rb); free(w); free(g); free(lam);
    return pot0b;
}

double orc_sens_poisson_adjoint(const double *eb, const orc_phys *ph, double *neb, double *nib) {
    return poisson_adjoint(eb, ph, neb, nib);
}

/* x adjoint of a CIC deposit at x: d/dx sum_k db[k] dens_k(x). */
static inline double deposit_gather(double x, const double *db, const orc_phys *ph) {
    const uint32_t n_g = ph->n_g;
    const double pos = x / ph->dx;
    int c = (int)pos;
    if (c > (int)n_g - 2) c = (int)n_g - 2;
    if (c < 0) c = 0;
    const double b0 = c == 0 ? 2.0 : 1.0, b1 = (c + 1 == (int)n_g - 1) ? 2.0 : 1.0;
    return ph->weight_factor_d / ph->dx * (b1 * db[c + 1] - b0 * db[c]);
}

/* Adjoint of a push of one particle (x, v) in field E with observable
 * weight wo (kind 0: <j E> term, 1: flux term), given the adjoints (xb, vb)
 * of the pushed state; returns the adjoints of (x, v) and adds the field's. */
static void push_adjoint(double x, double v, double f, double dt, const double *E, const orc_phys *ph, int kind,
                         double wo, double *xb, double *vb, double *eb) {
    const uint32_t n_g = ph->n_g;
    const double inv_dx = 1.0 / ph->dx;
    const double pos = x * inv_dx;
    int c = (int)pos;
    if (c > (int)n_g - 2) c = (int)n_g - 2;
    if (c < 0) c = 0;
    const double c2 = pos - c;
    const double ex = (1.0 - c2) * E[c] + c2 * E[c + 1];
    const double dex = (E[c + 1] - E[c]) * inv_dx;
    const double bt = *vb + dt * *xb; /* adjoint of the pushed velocity v + f ex */
    double nx = *xb;
    double nv = bt;
    double eg = bt * f; /* adjoint of ex */
    if (kind == 0) {
        const double q = v + f * ex;
        nv += wo * ex;
        eg += wo * q;
    } else if (c == (int)n_g - 2) {
        nv += wo * c2;
        nx += wo * v * inv_dx;
    }
    nx += eg * dex;
    eb[c] += eg * (1.0 - c2);
    eb[c + 1] += eg * c2;
    *xb = nx;
    *vb = nv;
}

/* Reverse sweep over the tape; returns d J / d voltage for the observable
 * weights (wP, wG).  horizon > 0: the adjoint restarts from zero at every
 * multiple of `horizon` steps (the sensitivity with the influence of the
 * voltage truncated to that many steps); 0: over the whole window. */
static double backward(const orc_phys *ph, tape_step *tape, uint32_t K, uint32_t cap, uint32_t horizon, double wP,
                       double wG) {
    const uint32_t n_g = ph->n_g;
    consts_f64 k;
    consts_init_f64(&k, ph);
    double *eb_[2][4], *eb = (double *)calloc(n_g, sizeof(double));
    for (int s = 0; s < 2; ++s)
        for (int c = 0; c < 4; ++c) eb_[s][c] = (double *)calloc(cap, sizeof(double));
    double *neb = (double *)calloc(n_g, sizeof(double)), *nib = (double *)calloc(n_g, sizeof(double));
    double *nib_acc = (double *)calloc(n_g, sizeof(double));
    double *xe = eb_[0][0], *ve[3] = {eb_[0][1], eb_[0][2], eb_[0][3]};
    double *xi = eb_[1][0], *vi[3] = {eb_[1][1], eb_[1][2], eb_[1][3]};
    double vbar = 0.0;
    const double fe = (double)ph->factor_e, fi = (double)ph->factor_i;
    const double dte = (double)ph->dt_e, dti = (double)ph->dt_i;
    for (int64_t t = (int64_t)K - 1; t >= 0; --t) {
        tape_step *ts = &tape[t];
        if (horizon && (uint64_t)(t + 1) % horizon == 0) /* a horizon ends after step t: restart the adjoint */
            for (int s = 0; s < 2; ++s)
                for (int c = 0; c < 4; ++c) memset(eb_[s][c], 0, sizeof(double) * cap);
        if (ts->ion) {
            for (uint32_t j = 0; j < ts->nri; ++j) {
                const rec_i *r = &ts->ri[j];
                double J[3][3];
                jac_i(r, J);
                const double w[3] = {vi[0][r->p], vi[1][r->p], vi[2][r->p]};
                for (int c = 0; c < 3; ++c) vi[c][r->p] = J[0][c] * w[0] + J[1][c] * w[1] + J[2][c] * w[2];
            }
        }
        for (uint32_t j = 0; j < ts->nre; ++j) {
            const rec_e *r = &ts->re[j];
            double J[3][3], Jc[3][3];
            jac_e(&k, r, J, Jc);
            const uint32_t p = r->p;
            const double w[3] = {ve[0][p], ve[1][p], ve[2][p]};
            double nv[3];
            for (int c = 0; c < 3; ++c) nv[c] = J[0][c] * w[0] + J[1][c] * w[1] + J[2][c] * w[2];
            if (r->ev == 3 && r->ce != SENS_NO_SLOT) {
                const uint32_t s = r->ce;
                const double wc[3] = {ve[0][s], ve[1][s], ve[2][s]};
                for (int c = 0; c < 3; ++c) nv[c] += Jc[0][c] * wc[0] + Jc[1][c] * wc[1] + Jc[2][c] * wc[2];
                xe[p] += xe[s];
                xe[s] = ve[0][s] = ve[1][s] = ve[2][s] = 0.0;
            }
            if (r->ev == 3 && r->ci != SENS_NO_SLOT) {
                const uint32_t s = r->ci;
                xe[p] += xi[s];
                xi[s] = vi[0][s] = vi[1][s] = vi[2][s] = 0.0;
            }
            for (int c = 0; c < 3; ++c) ve[c][p] = nv[c];
        }
        memset(eb, 0, sizeof(double) * n_g);
        for (uint32_t p = 0; p < ts->ne; ++p) {
            if (!(ts->xe[p] >= 0.0)) continue;
            push_adjoint(ts->xe[p], ts->vxe[p], fe, dte, ts->E, ph, 0, wP, &xe[p], &ve[0][p], eb);
        }
        if (ts->ion) {
            for (uint32_t p = 0; p < ts->ni; ++p) {
                if (!(ts->xi[p] >= 0.0)) continue;
                push_adjoint(ts->xi[p], ts->vxi[p], fi, dti, ts->E, ph, 1, wG, &xi[p], &vi[0][p], eb);
            }
        }
        vbar += ts->cosv * poisson_adjoint(eb, ph, neb, nib);
        for (uint32_t p = 0; p < ts->ne; ++p)
            if (ts->xe[p] >= 0.0) xe[p] += deposit_gather(ts->xe[p], neb, ph);
        for (uint32_t j = 0; j < n_g; ++j) nib_acc[j] += nib[j];
        if (ts->ion) {
            for (uint32_t p = 0; p < ts->ni; ++p)
                if (ts->xi[p] >= 0.0) xi[p] += deposit_gather(ts->xi[p], nib_acc, ph);
            memset(nib_acc, 0, sizeof(double) * n_g);
        }
    }
    for (int s = 0; s < 2; ++s)
        for (int c = 0; c < 4; ++c) free(eb_[s][c]);
    free(eb); free(neb); free(nib); free(nib_acc);
    return vbar;
}

/* ------------------------------------------------------------------ */
/* entry point                                                         */
/* ------------------------------------------------------------------ */

/* Observable normalisations: per unit of the raw sums. */
static void obs_scale(const orc_phys *ph, uint32_t K, double *cP, double *cG) {
    const double w_over_a = ph->weight_factor_d * ph->dx;
    uint32_t k_i = 0;
    for (uint32_t t = 0; t < K; ++t) k_i += (t % ph->n_sub) == 0;
    *cP = -ORC_E_CHARGE * w_over_a / ((double)ph->gap) / (double)K;
    *cG = 2.0 * ph->weight_factor_d / (double)(k_i ? k_i : 1);
}

int orc_sens_run(const orc_phys *ph, const float *sig_e, const float *sig_i, const float *cs, double voltage,
                 uint32_t steps, uint32_t horizon, int f64, orc_sens_io *io, double obs[2], double grad[2]) {
    const uint32_t cap = io->capacity, n_g = ph->n_g;
    if (ph->n_t == 0 || ph->n_sub == 0 || n_g < 3 || io->n[0] > cap || io->n[1] > cap) return -1;
    if (horizon % ph->n_sub) return -1;
    tape_step *tape = grad ? (tape_step *)calloc(steps ? steps : 1, sizeof(tape_step)) : NULL;
    double raw[2] = {0.0, 0.0};
    uint32_t dev_err = 0;
    if (!f64) {
        sp_f32 s[2];
        for (int k = 0; k < 2; ++k) {
            s[k].x = io->x[k]; s[k].vx = io->vx[k]; s[k].vy = io->vy[k]; s[k].vz = io->vz[k];
            for (int c = 0; c < 4; ++c) s[k].r[c] = io->rng[k][c];
            s[k].n = io->n[k];
            s[k].cap = cap;
        }
        float *de = (float *)calloc(n_g, sizeof(float)), *di = (float *)calloc(n_g, sizeof(float));
        float *E = (float *)calloc(n_g, sizeof(float));
        for (uint32_t t = 0; t < steps; ++t)
            step_f32(&s[0], &s[1], de, di, E, ph, sig_e, sig_i, cs, voltage, t, raw, tape ? &tape[t] : NULL,
                     &dev_err);
        io->n[0] = s[0].n;
        io->n[1] = s[1].n;
        free(de); free(di); free(E);
    } else {
        sp_f64 s[2];
        for (int k = 0; k < 2; ++k) {
            double **pl[4] = {&s[k].x, &s[k].vx, &s[k].vy, &s[k].vz};
            float *src[4] = {io->x[k], io->vx[k], io->vy[k], io->vz[k]};
            for (int c = 0; c < 4; ++c) {
                *pl[c] = (double *)calloc(cap, sizeof(double));
                for (uint32_t p = 0; p < io->n[k]; ++p) (*pl[c])[p] = (double)src[c][p];
            }
            for (int c = 0; c < 4; ++c) s[k].r[c] = io->rng[k][c];
            s[k].n = io->n[k];
            s[k].cap = cap;
        }
        double *de = (double *)calloc(n_g, sizeof(double)), *di = (double *)calloc(n_g, sizeof(double));
        double *E = (double *)calloc(n_g, sizeof(double));
        for (uint32_t t = 0; t < steps; ++t)
            step_f64(&s[0], &s[1], de, di, E, ph, sig_e, sig_i, cs, voltage, t, raw, tape ? &tape[t] : NULL,
                     &dev_err);
        for (int k = 0; k < 2; ++k) {
            double *pl[4] = {s[k].x, s[k].vx, s[k].vy, s[k].vz};
            float *dst[4] = {io->x[k], io->vx[k], io->vy[k], io->vz[k]};
            for (int c = 0; c < 4; ++c) {
                for (uint32_t p = 0; p < s[k].n; ++p) dst[c][p] = (float)pl[c][p];
                free(pl[c]);
            }
            io->n[k] = s[k].n;
        }
        free(de); free(di); free(E);
    }
    double cP, cG;
    obs_scale(ph, steps, &cP, &cG);
    obs[0] = cP * raw[0];
    obs[1] = cG * raw[1];
    io->dev_err = dev_err;
    if (grad) {
        grad[0] = backward(ph, tape, steps, cap, horizon, cP, 0.0);
        grad[1] = backward(ph, tape, steps, cap, horizon, 0.0, cG);
        for (uint32_t t = 0; t < steps; ++t) tape_free(&tape[t]);
        free(tape);
    }
    return 0;
}
