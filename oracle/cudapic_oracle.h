/*
 * cudapic_oracle.h -- CPU restatement of the cudaPIC per-timestep PIC/MCC cycle.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * cudapic_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product library never links or calls it.
 *
 * Every function restates the arithmetic of one reference kernel or host
 * helper (cited per function, paths relative to the reference project), in
 * plain C with IEEE float semantics (compiled with -ffp-contract=off so that
 * a*b+c is never fused unless written as fmaf).  Transcendentals follow the
 * same published methods as the CUDA kernels (Cody-Waite argument reduction
 * plus Taylor / atanh series, see cudapic_oracle_math.c) so that collision
 * decisions and post-collision velocities can be compared bit-exactly; the
 * CPU tests separately bound those functions against libm in double.
 *
 * FP64 references of the eduPIC code (C/eduPIC.cc) are provided for the
 * deposit and the Poisson solve, the tolerance targets of the f32 kernels.
 */
#ifndef CUDAPIC_ORACLE_H
#define CUDAPIC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Physical constants, Rust-CUDA/src/main.rs:30-37 (same values as C/eduPIC.cc:36-45). */
#define ORC_PI          3.141592653589793
#define ORC_E_CHARGE    1.60217662e-19
#define ORC_E_MASS      9.10938356e-31
#define ORC_AR_MASS     6.63352090e-26
#define ORC_K_BOLTZMANN 1.38064852e-23
#define ORC_EPSILON0    8.85418781e-12
#define ORC_CS_RANGES   1000000
#define ORC_N_EEPF      2000
#define ORC_N_IFED      200

/* Runtime replacement of the reference's compile-time simulation constants
 * (Rust-CUDA/src/main.rs:40-50, 53-59, 79-82). */
typedef struct orc_params {
    uint32_t n_g;
    uint32_t n_t;
    uint32_t n_sub;
    uint32_t capacity;
    double frequency;
    double voltage;
    double gap;
    double pressure;
    double temperature;
    double weight;
    double electrode_area;
} orc_params;

/* Derived f32/f64 constants exactly as the reference forms them
 * (`X as Real` casts of f64 expressions, Rust-CUDA/src/main.rs:53-109). */
typedef struct orc_phys {
    uint32_t n_g;
    uint32_t capacity;
    float inv_dx;            /* INV_DX as Real                          */
    float weight_factor;     /* WEIGHT_FACTOR as Real                   */
    float gap;               /* L as Real                               */
    float dt_e, dt_i;        /* DT_E, DT_I as Real                      */
    float factor_e, factor_i;/* FACTOR_E, FACTOR_I as Real              */
    float e_charge;          /* E_CHARGE_F                              */
    float alpha;             /* ALPHA_F = -DX^2/eps0                    */
    float half_dx_over_eps;  /* HALF_DX_OVER_EPS_F                      */
    float half_inv_dx;       /* HALF_INV_DX_F                           */
    float normal_range;      /* sqrt(kT/M_Ar) as Real                   */
    float f1, f2;            /* F1, F2                                  */
    float half_me_over_e;    /* HALF_E_MASS_OVER_E_CHARGE               */
    float half_mu_over_e;    /* HALF_MU_ARAR_OVER_E_CHARGE              */
    float min_x, max_x;      /* MIN_X_F, MAX_X_F (EEPF window)          */
    float eepf_half_kick;    /* (DT_E*E_CHARGE/E_MASS) as Real          */
    double dx;
    double weight_factor_d;  /* WEIGHT/(A*DX) in double (eduPIC FACTOR_W) */
    double gas_density;
    double dt_e_d, dt_i_d;
    double voltage;
    double omega;            /* 2 pi f */
    uint32_t n_t, n_sub;
} orc_phys;

void orc_params_default(orc_params *p);
void orc_phys_from_params(const orc_params *p, orc_phys *out);

/* ---- RNG: xoshiro128+ (Rust-CUDA/src/main.rs:860-906, 1446-1496) ---- */
uint32_t orc_xoshiro128p_next(uint32_t s[4]);
void orc_xoshiro128p_stream(const uint32_t seed[4], uint32_t n, uint32_t *out);
float orc_u32_to_real(uint32_t x);
void orc_jump(uint32_t s[4]);
/* Stream k = master after k jumps; writes the four state planes. */
int orc_seed_streams(const uint32_t master[4], uint32_t n,
                     uint32_t *s0, uint32_t *s1, uint32_t *s2, uint32_t *s3);

/* ---- transcendental functions (published methods, see the .c file) ---- */
float orc_expf(float x);
float orc_logf(float x);
float orc_sinf(float x);
float orc_cosf(float x);
float orc_tanf(float x);
float orc_atanf(float x);
float orc_atan2f(float y, float x);
float orc_acosf(float x);
/* Apply function `fn` (0 exp, 1 log, 2 sin, 3 cos, 4 tan, 5 atan, 6 acos,
 * 7 atan2 with y=in, x=in2) elementwise. */
void orc_math_apply(int fn, const float *in, const float *in2, float *out, uint32_t n);

/* ---- cross sections (Rust-CUDA/src/main.rs:1378-1444) ---- */
void orc_cross_sections(double gas_density, float *cs /* 5*CS_RANGES */,
                        float *sigma_tot_e, float *sigma_tot_i);

/* ---- deposition ---- */
/* f32 restatement of get_density (Rust-CUDA/src/main.rs:356-406), sequential order. */
void orc_get_density_f32(const float *x, uint32_t n, float *density, const orc_phys *ph);
/* FP64 deposit of eduPIC (C/eduPIC.cc:520-529); density is overwritten. */
void orc_get_density_f64(const float *x, uint32_t n, double *density, const orc_phys *ph);

/* ---- Poisson ---- */
/* FP64 Thomas solve + field of eduPIC (C/eduPIC.cc:461-494) from f32 densities. */
void orc_poisson_thomas_f64(const float *e_density, const float *i_density, double pot0,
                            double *pot, double *efield, const orc_phys *ph);
/* f32 restatement of solve_poisson_scan_f32 (Rust-CUDA/src/main.rs:408-494), sequential scans. */
void orc_poisson_scan_f32(const float *e_density, const float *i_density, float pot0,
                          float *pot, float *efield, const orc_phys *ph);
/* solve_poisson_dps_flexible (Rust-CUDA/src/main.rs:496-564) in double. */
void orc_poisson_dps_flexible_f64(const double *source, double *pot, uint32_t n,
                                  double psi_left, double psi_right, double dx);

/* ---- push + absorb + compact (Rust-CUDA/src/main.rs:566-678), stable order ---- */
void orc_wall_count(const float *efield, const float *sx, const float *svx, const float *svy, const float *svz,
                    uint32_t n, float factor, float dt, const orc_phys *ph, int ions, uint64_t counts[2],
                    uint32_t *ifed_pow, uint32_t *ifed_gnd);
uint32_t orc_move_and_compact(const float *efield,
                              const float *sx, const float *svx, const float *svy, const float *svz,
                              float *dx_, float *dvx, float *dvy, float *dvz,
                              uint32_t n, float factor, float dt, const orc_phys *ph,
                              uint32_t *src_index /* may be NULL: survivor's source index */);

/* ---- MCC (Rust-CUDA/src/main.rs:971-1292) ----
 * Particles are processed in index order; spawns are appended in that order.
 * events[i] (may be NULL): 0 none, 1 elastic, 2 excitation, 3 ionization
 * (electrons); 0 none, 4 isotropic, 5 backscatter (ions).
 * *n_e / *n_i are updated with the spawns; spawns beyond capacity are dropped
 * and counted in *dropped. */
void orc_check_collisions_e(const float *sigma_tot_e, const float *cs, uint32_t n_active,
                            float *x, float *vx, float *vy, float *vz,
                            uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3,
                            float *ix, float *ivx, float *ivy, float *ivz,
                            uint32_t *n_e, uint32_t *n_i, const orc_phys *ph,
                            uint8_t *events, uint32_t *dropped);
/* The same with the fused step's scattering arithmetic: the sines and
 * cosines of the Euler angles, of chi = acos(c) and of eta + pi from their
 * algebraic forms instead of evaluating the angles (same draws and events;
 * velocities within the rounding of the skipped transcendentals). */
void orc_check_collisions_e_alg(const float *sigma_tot_e, const float *cs, uint32_t n_active,
                                float *x, float *vx, float *vy, float *vz,
                                uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3,
                                float *ix, float *ivx, float *ivy, float *ivz,
                                uint32_t *n_e, uint32_t *n_i, const orc_phys *ph,
                                uint8_t *events, uint32_t *dropped);
void orc_check_collisions_i(const float *sigma_tot_i, const float *cs, uint32_t n_active,
                            float *vx, float *vy, float *vz,
                            uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3,
                            const orc_phys *ph, uint8_t *events);
/* Decide-only helper: collision probability of an electron / ion computed in
 * double with libm (used to bound the ambiguity band of the f32 decision). */
double orc_p_coll_e_exact(const float *sigma_tot_e, float vx, float vy, float vz, const orc_phys *ph);

/* ---- diagnostics (Rust-CUDA/src/main.rs:1294-1339) ---- */
void orc_accumulate_density(const float *density, double *cumul, uint32_t n_g);
void orc_accumulate_eepf(const float *x, const float *vx, const float *vy, const float *vz,
                         const float *efield, uint32_t n_active, uint32_t *eepf,
                         const orc_phys *ph);

/* ---- XT diagnostics (C/eduPIC.cc:557-576, :599-614) ---- */
/* One step of eduPIC's measurement branch for one species, before the push,
 * in the f32 arithmetic of the GPU kernel: with c1 = 1 - c2 and c2 the CIC
 * weights of node p and p + 1, v = vx + 1/2 factor e_x and E = 1/2 m |v|^2 / e,
 * out[q * n_g + node] += c (q 0), c v (q 1), c E (q 2) and, for electrons,
 * c sigma_ion(E) |v| DT_E n_gas (q 3, cs_ion: eduPIC's sigma[E_ION] table). */
void orc_xt_accumulate(const float *efield, const float *x, const float *vx, const float *vy, const float *vz,
                       uint32_t n, int ions, const float *cs_ion, const orc_phys *ph, double *out);


/* ---- voltage sensitivity (cudapic_oracle_sens.c) ---- */
/* Particles of both species in their slots ([0] electrons, [1] ions):
 * positions (dead slots x = -1), velocities, the four RNG planes, the slot
 * counts n and the common capacity; dev_err receives 0x1 / 0x2 when an
 * electron / ion spawn found no slot. */
typedef struct orc_sens_io {
    float *x[2], *vx[2], *vy[2], *vz[2];
    uint32_t *rng[2][4];
    uint32_t n[2];
    uint32_t capacity;
    uint32_t dev_err;
} orc_sens_io;
/* Runs `steps` steps of the slot-form model from step 0 of the RF period at
 * amplitude `voltage`, in place; obs = (J_P [W m^-3], J_G [m^-2 s^-1]).
 * f64 = 0: the f32 arithmetic of the CUDA path; 1: the same model in double.
 * grad (may be NULL): d obs / d voltage by the pathwise adjoint; horizon
 * (a multiple of N_SUB, 0 = the whole window): the adjoint restarts from
 * zero every `horizon` steps.  Returns -1 on bad arguments. */
/* Adjoint of the Poisson solve and field (the closed form of the CUDA solve,
 * C/eduPIC.cc:461-494): from the field adjoint eb [n_g], the adjoints of
 * the electron and ion densities; returns the adjoint of pot0. */
double orc_sens_poisson_adjoint(const double *eb, const orc_phys *ph, double *neb, double *nib);
int orc_sens_run(const orc_phys *ph, const float *sigma_tot_e, const float *sigma_tot_i, const float *cs,
                 double voltage, uint32_t steps, uint32_t horizon, int f64, orc_sens_io *io, double obs[2],
                 double grad[2]);

#ifdef __cplusplus
}
#endif
#endif
