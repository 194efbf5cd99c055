/*
 * edupic_hooks.h -- force-included into the reference CPU build of eduPIC
 * (see Makefile / edupic.sed).  Test and baseline infrastructure only.
 *
 * Defaults reproduce the original constants of C/eduPIC.cc:49-58, 89.
 * EDUPIC_STEP_HOOK counts particle-steps exactly as the GPU metric does
 * (every electron each step, every ion on steps t % N_SUB == 0) and, every
 * EDUPIC_MARK_EVERY steps, prints a line
 *     EDUPIC_MARK <steps> <particle_steps> <CLOCK_MONOTONIC ns>
 * to stderr so that a driver can time any window of the run.
 */
#include <cstdio>
#include <cstdlib>
#include <ctime>

// Grid and time resolution size static arrays: compile-time.  Voltage, gap,
// pressure, superparticle weight and the random seed are read from the
// environment (EDUPIC_VOLTAGE, EDUPIC_L, EDUPIC_PRESSURE, EDUPIC_WEIGHT,
// EDUPIC_SEED) when set.
static inline double edupic_env(const char *name, double def) {
    const char *v = getenv(name);
    return v ? atof(v) : def;
}

#ifndef EDUPIC_N_G
#define EDUPIC_N_G 400
#endif
#ifndef EDUPIC_N_T
#define EDUPIC_N_T 4000
#endif
#ifndef EDUPIC_VOLTAGE
#define EDUPIC_VOLTAGE edupic_env("EDUPIC_VOLTAGE", 250.0)
#endif
#ifndef EDUPIC_L
#define EDUPIC_L edupic_env("EDUPIC_L", 0.025)
#endif
#ifndef EDUPIC_PRESSURE
#define EDUPIC_PRESSURE edupic_env("EDUPIC_PRESSURE", 10.0)
#endif
#ifndef EDUPIC_WEIGHT
#define EDUPIC_WEIGHT edupic_env("EDUPIC_WEIGHT", 7.0e4)
#endif
#ifndef EDUPIC_N_INIT
#define EDUPIC_N_INIT 1000
#endif
#ifndef EDUPIC_MAX_N_P
#define EDUPIC_MAX_N_P 8388608
#endif
// Mersenne-Twister seed of the run (C/eduPIC.cc:165 seeds from
// std::random_device): EDUPIC_SEED from the environment, default 5489.
#ifndef EDUPIC_SEED
#define EDUPIC_SEED ((unsigned)edupic_env("EDUPIC_SEED", 5489.0))
#endif
#ifndef EDUPIC_STEPS_PER_CYCLE
#define EDUPIC_STEPS_PER_CYCLE N_T
#endif
#ifndef EDUPIC_MARK_EVERY
#define EDUPIC_MARK_EVERY 1000
#endif

static unsigned long long edupic_steps_done = 0;
static unsigned long long edupic_particle_steps = 0;

static inline unsigned long long edupic_now_ns() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (unsigned long long)ts.tv_sec * 1000000000ull + (unsigned long long)ts.tv_nsec;
}

// Start barrier of a group of processes timed together: with
// EDUPIC_READY_FILE and EDUPIC_START_FILE set, the first time step (after the
// cross sections are set up and picdata.bin is read) creates the ready file
// and waits until the start file exists (at most ten minutes).
static inline void edupic_start_barrier() {
    const char *ready = getenv("EDUPIC_READY_FILE");
    const char *start = getenv("EDUPIC_START_FILE");
    if (!ready || !start) return;
    if (FILE *f = fopen(ready, "w")) fclose(f);
    const unsigned long long t0 = edupic_now_ns();
    for (;;) {
        if (FILE *f = fopen(start, "r")) {
            fclose(f);
            return;
        }
        if (edupic_now_ns() - t0 > 600ull * 1000000000ull) return;
        struct timespec ts = {0, 200000};
        nanosleep(&ts, nullptr);
    }
}

static inline void edupic_hook_step(int t, int n_e, int n_i, int n_sub) {
    if (edupic_steps_done == 0) edupic_start_barrier();
    if (edupic_steps_done % EDUPIC_MARK_EVERY == 0)
        fprintf(stderr, "EDUPIC_MARK %llu %llu %llu\n", edupic_steps_done, edupic_particle_steps,
                edupic_now_ns());
    edupic_particle_steps += (unsigned long long)n_e + ((t % n_sub) == 0 ? (unsigned long long)n_i : 0ull);
    ++edupic_steps_done;
}

__attribute__((destructor)) static void edupic_report_end() {
    fprintf(stderr, "EDUPIC_MARK %llu %llu %llu\n", edupic_steps_done, edupic_particle_steps,
            edupic_now_ns());
}

#define EDUPIC_STEP_HOOK(t) edupic_hook_step((t), N_e, N_i, N_SUB)
