// host.cpp -- parameters, derived constants, error reporting, launch-config
// caches and the cross-section tables of libcudapic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace cudapic {

namespace {
thread_local std::string g_last_error;

constexpr double PI = 3.141592653589793;       // Rust-CUDA/src/main.rs:30
constexpr double E_CHARGE = 1.60217662e-19;    // :32
constexpr double E_MASS = 9.10938356e-31;      // :33
constexpr double AR_MASS = 6.63352090e-26;     // :34
constexpr double K_BOLTZMANN = 1.38064852e-23; // :36
constexpr double EPSILON0 = 8.85418781e-12;    // :37

struct DeviceInfo {
    int sms = 0;
    int smem_optin = 0;
};
std::mutex g_dev_mu;
DeviceInfo g_dev[64];

DeviceInfo &device_info() {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_dev_mu);
    DeviceInfo &d = g_dev[dev & 63];
    if (d.sms == 0) {
        cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (d.sms <= 0) d.sms = 1;
    }
    return d;
}
}  // namespace

int fail(int status, const std::string &msg) {
    g_last_error = msg;
    return status;
}

int check_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return CUDAPIC_OK;
    return fail(CUDAPIC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_launch(const char *kernel) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return CUDAPIC_OK;
    return fail(CUDAPIC_ERR_CUDA, std::string("launch ") + kernel + ": " + cudaGetErrorString(e));
}

int sm_count() { return device_info().sms; }
int max_smem_optin() { return device_info().smem_optin; }

namespace {
// Built-in launch shapes (chosen with cudapic_b200.autotune on B200).
constexpr cudapic_tuning kDefaultTuning = {
    /*density_threads*/ 512, /*density_ctas_per_sm*/ 4, /*density_copies*/ 4, /*density_cluster*/ 4,
    /*push_stages*/ 2, /*push_ctas_per_sm*/ 4,
    /*mcc_stages*/ 2, /*mcc_ctas_per_sm*/ 4, /*mcc_variant*/ 1,
    /*step_stages*/ 2, /*step_ctas_per_sm*/ 3, /*step_rows*/ 2,
    /*inplace_ctas_per_sm*/ 4, /*inplace_copies*/ 4, /*inplace_prefetch*/ 1,
    /*scatter_ctas_per_sm*/ 4};
std::mutex g_tune_mu;
cudapic_tuning g_tuning = kDefaultTuning;
uint64_t g_tuning_gen = 0;  // advanced by every cudapic_set_tuning
}  // namespace

namespace {
thread_local bool t_pdl = false;
}

bool pdl_enabled() { return t_pdl; }
PdlScope::PdlScope(bool on) : prev(t_pdl) { t_pdl = on; }
PdlScope::~PdlScope() { t_pdl = prev; }

cudapic_tuning tuning() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return g_tuning;
}

uint64_t tuning_generation() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return g_tuning_gen;
}

unsigned persistent_grid(int per_sm, uint64_t units) {
    const uint64_t cap = (uint64_t)sm_count() * (uint64_t)std::max(per_sm, 1);
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(cap, units));
}

int validate_grid(const cudapic_grid *g) {
    if (!g) return fail(CUDAPIC_ERR_ARG, "grid is null");
    if (g->n_g < 3 || g->n_g > 16384) return fail(CUDAPIC_ERR_ARG, "grid.n_g must be in [3, 16384]");
    if (g->capacity == 0) return fail(CUDAPIC_ERR_ARG, "grid.capacity must be > 0");
    if (g->n_t == 0 || g->n_sub == 0) return fail(CUDAPIC_ERR_ARG, "grid.n_t and grid.n_sub must be > 0");
    return CUDAPIC_OK;
}

}  // namespace cudapic

using namespace cudapic;

extern "C" void cudapic_params_default(cudapic_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // Rust-CUDA/src/main.rs:40-50, 79
    p->n_g = 400;
    p->n_t = 4000;
    p->n_sub = 20;
    p->capacity = 120000;
    p->frequency = 13.56e6;
    p->voltage = 250.0;
    p->gap = 0.025;
    p->pressure = 10.0;
    p->temperature = 350.0;
    p->weight = 7.0e4;
    p->electrode_area = 1.0e-4;
    p->flags = 0;
}

// Every `X as Real` constant of Rust-CUDA/src/main.rs:53-109 is the double
// expression rounded to float once.
extern "C" int cudapic_grid_from_params(const cudapic_params *p, cudapic_grid *o) {
    if (!p || !o) return fail(CUDAPIC_ERR_ARG, "grid_from_params: null pointer");
    if (p->n_g < 3 || p->n_g > 16384) return fail(CUDAPIC_ERR_ARG, "params.n_g must be in [3, 16384]");
    if (p->n_t == 0 || p->n_sub == 0) return fail(CUDAPIC_ERR_ARG, "params.n_t and n_sub must be > 0");
    if (p->capacity == 0 || p->capacity > (1u << 28))
        return fail(CUDAPIC_ERR_ARG, "params.capacity must be in [1, 2^28]");
    if (!(p->frequency > 0) || !(p->gap > 0) || !(p->pressure > 0) || !(p->temperature > 0) ||
        !(p->weight > 0) || !(p->electrode_area > 0))
        return fail(CUDAPIC_ERR_ARG, "params: physical parameters must be positive");
    std::memset(o, 0, sizeof(*o));
    const double period = 1.0 / p->frequency;
    const double dt_e = period / (double)p->n_t;
    const double dt_i = (double)p->n_sub * dt_e;
    const double dx = p->gap / (double)(p->n_g - 1);
    const double inv_dx = 1.0 / dx;
    o->n_g = p->n_g;
    o->capacity = p->capacity;
    o->n_t = p->n_t;
    o->n_sub = p->n_sub;
    o->flags = p->flags;
    o->inv_dx = (float)inv_dx;
    o->weight_factor = (float)(p->weight / (p->electrode_area * dx));
    o->gap = (float)p->gap;
    o->dt_e = (float)dt_e;
    o->dt_i = (float)dt_i;
    o->factor_e = (float)(dt_e / E_MASS * (-E_CHARGE));
    o->factor_i = (float)(dt_i / AR_MASS * E_CHARGE);
    o->e_charge = (float)E_CHARGE;
    o->alpha = (float)(-dx * dx / EPSILON0);
    o->half_dx_over_eps = (float)(dx / (2.0 * EPSILON0));
    o->half_inv_dx = (float)(0.5 * inv_dx);
    o->normal_range = (float)std::sqrt(K_BOLTZMANN * p->temperature / AR_MASS);
    o->f1 = (float)(E_MASS / (E_MASS + AR_MASS));
    o->f2 = (float)(AR_MASS / (E_MASS + AR_MASS));
    o->half_me_over_e = (float)(0.5 * E_MASS / E_CHARGE);
    o->half_mu_over_e = (float)(0.5 * (AR_MASS / 2.0) / E_CHARGE);
    o->min_x = (float)(0.45 * p->gap);
    o->max_x = (float)(0.55 * p->gap);
    o->eepf_half_kick = (float)(dt_e * E_CHARGE / E_MASS);
    o->dx = dx;
    o->weight_factor_d = p->weight / (p->electrode_area * dx);
    o->gas_density = p->pressure / (K_BOLTZMANN * p->temperature);
    o->voltage = p->voltage;
    o->dev_err = nullptr;
    o->work = nullptr;
    return CUDAPIC_OK;
}

extern "C" const char *cudapic_status_string(int s) {
    switch (s) {
    case CUDAPIC_OK: return "ok";
    case CUDAPIC_ERR_CUDA: return "CUDA error";
    case CUDAPIC_ERR_CAPACITY: return "particle capacity exceeded";
    case CUDAPIC_ERR_ARG: return "invalid argument";
    case CUDAPIC_ERR_TIMEOUT: return "device wait timed out";
    case CUDAPIC_ERR_NOT_SUPPORTED: return "not supported on this device";
    case CUDAPIC_ERR_STATE: return "invalid state";
    default: return "unknown status";
    }
}

extern "C" const char *cudapic_last_error(void) { return g_last_error.c_str(); }

extern "C" int cudapic_get_tuning(cudapic_tuning *out) {
    if (!out) return fail(CUDAPIC_ERR_ARG, "get_tuning: null pointer");
    *out = tuning();
    return CUDAPIC_OK;
}

extern "C" int cudapic_set_tuning(const cudapic_tuning *t) {
    if (!t) return fail(CUDAPIC_ERR_ARG, "set_tuning: null pointer");
    cudapic_tuning v = *t;
    const cudapic_tuning d = kDefaultTuning;
    if (!v.density_threads) v.density_threads = d.density_threads;
    if (!v.density_ctas_per_sm) v.density_ctas_per_sm = d.density_ctas_per_sm;
    if (!v.density_copies) v.density_copies = d.density_copies;
    if (!v.density_cluster) v.density_cluster = d.density_cluster;
    if (!v.push_stages) v.push_stages = d.push_stages;
    if (!v.push_ctas_per_sm) v.push_ctas_per_sm = d.push_ctas_per_sm;
    if (!v.mcc_stages) v.mcc_stages = d.mcc_stages;
    if (!v.mcc_ctas_per_sm) v.mcc_ctas_per_sm = d.mcc_ctas_per_sm;
    if (!v.mcc_variant) v.mcc_variant = d.mcc_variant;
    if (!v.step_stages) v.step_stages = d.step_stages;
    if (!v.step_ctas_per_sm) v.step_ctas_per_sm = d.step_ctas_per_sm;
    if (!v.step_rows) v.step_rows = d.step_rows;
    if (!v.inplace_ctas_per_sm) v.inplace_ctas_per_sm = d.inplace_ctas_per_sm;
    if (!v.inplace_copies) v.inplace_copies = d.inplace_copies;
    if (!v.inplace_prefetch) v.inplace_prefetch = d.inplace_prefetch;
    if (!v.scatter_ctas_per_sm) v.scatter_ctas_per_sm = d.scatter_ctas_per_sm;
    const bool ok = (v.density_threads == 256 || v.density_threads == 512 || v.density_threads == 1024) &&
                    v.density_ctas_per_sm >= 1 && v.density_ctas_per_sm <= 8 && v.density_copies >= 1 &&
                    v.density_copies <= 32 &&
                    (v.density_cluster == 1 || v.density_cluster == 2 || v.density_cluster == 4 ||
                     v.density_cluster == 8) &&
                    v.push_stages >= 2 && v.push_stages <= 6 && v.push_ctas_per_sm >= 1 && v.push_ctas_per_sm <= 8 &&
                    v.mcc_stages >= 2 && v.mcc_stages <= 4 && v.mcc_ctas_per_sm >= 1 && v.mcc_ctas_per_sm <= 8 &&
                    (v.mcc_variant == 1 || v.mcc_variant == 2) && v.step_stages >= 2 && v.step_stages <= 6 &&
                    v.step_ctas_per_sm >= 1 && v.step_ctas_per_sm <= 8 &&
                    (v.step_rows == 1 || v.step_rows == 2 || v.step_rows == 4) && v.inplace_ctas_per_sm >= 1 &&
                    v.inplace_ctas_per_sm <= 8 && (v.inplace_copies == -1 || (v.inplace_copies >= 1 && v.inplace_copies <= 8)) &&
                    (v.inplace_prefetch == -1 || (v.inplace_prefetch >= 1 && v.inplace_prefetch <= 4)) &&
                    v.scatter_ctas_per_sm >= 1 && v.scatter_ctas_per_sm <= 8;
    if (!ok) return fail(CUDAPIC_ERR_ARG, "set_tuning: value out of range");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuning = v;
    ++g_tuning_gen;
    return CUDAPIC_OK;
}

extern "C" int cudapic_version(void) { return CUDAPIC_VERSION; }

// ---------------------------------------------------------------------
// Cross sections, Rust-CUDA/src/main.rs:1378-1444 (Phelps fits evaluated in
// double with the C library's pow/exp/sqrt, rounded to float; totals are the
// double sum of the float entries times the gas density, rounded to float).
// ---------------------------------------------------------------------
namespace {

double q_mom_e(double e) {
    return 1.0e-20 * (std::fabs(6.0 / std::pow(1.0 + e / 0.1 + std::pow(e / 0.6, 2.0), 3.3) -
                                1.1 * std::pow(e, 1.4) / (1.0 + std::pow(e / 15.0, 1.2)) /
                                    std::sqrt(1.0 + std::pow(e / 5.5, 2.5) + std::pow(e / 60.0, 4.1))) +
                      0.05 / std::pow(1.0 + e / 10.0, 2.0) + 0.01 * std::pow(e, 3.0) / (1.0 + std::pow(e / 12.0, 6.0)));
}

double q_exc_e(double e) {
    if (e <= 11.5) return 0.0;
    return (0.034 * std::pow(e - 11.5, 1.1) * (1.0 + std::pow(e / 15.0, 2.8)) / (1.0 + std::pow(e / 23.0, 5.5)) +
            0.023 * (e - 11.5) / std::pow(1.0 + e / 80.0, 1.9)) *
           1.0e-20;
}

double q_ion_e(double e) {
    if (e <= 15.8) return 0.0;
    return (970.0 * (e - 15.8) / std::pow(70.0 + e, 2.0) + 0.06 * std::pow(e - 15.8, 2.0) * std::exp(-e / 9.0)) *
           1.0e-20;
}

double q_moi(double e_lab) { return 1.15e-18 * std::pow(e_lab, -0.1) * std::pow(1.0 + 0.015 / e_lab, 0.6); }
double q_iso(double e_lab) {
    return 2.0e-19 * std::pow(e_lab, -0.5) / (1.0 + e_lab) + 3.0e-19 * e_lab / std::pow(1.0 + e_lab / 3.0, 2.0);
}
double q_chx(double e_lab) { return 0.5 * (q_moi(e_lab) - q_iso(e_lab)); }

void cs_range(double gas_density, float *cs, float *se, float *si, uint32_t lo, uint32_t hi) {
    const uint32_t R = CUDAPIC_CS_RANGES;
    for (uint32_t i = lo; i < hi; ++i) {
        const double e = (i == 0) ? 0.001 : (double)i * 0.001;
        const float a = (float)q_mom_e(e), b = (float)q_exc_e(e), c = (float)q_ion_e(e);
        const float d = (float)q_iso(2.0 * e), f = (float)q_chx(2.0 * e);
        cs[0 * R + i] = a;
        cs[1 * R + i] = b;
        cs[2 * R + i] = c;
        cs[3 * R + i] = d;
        cs[4 * R + i] = f;
        se[i] = (float)(((double)a + (double)b + (double)c) * gas_density);
        si[i] = (float)(((double)d + (double)f) * gas_density);
    }
}

}  // namespace

extern "C" int cudapic_cross_sections(double gas_density, float *cs, float *sigma_tot_e, float *sigma_tot_i) {
    if (!cs || !sigma_tot_e || !sigma_tot_i) return fail(CUDAPIC_ERR_ARG, "cross_sections: null pointer");
    if (!(gas_density > 0)) return fail(CUDAPIC_ERR_ARG, "cross_sections: gas density must be positive");
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const uint32_t R = CUDAPIC_CS_RANGES;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t) {
        uint32_t lo = (uint32_t)((uint64_t)R * t / nt), hi = (uint32_t)((uint64_t)R * (t + 1) / nt);
        pool.emplace_back(cs_range, gas_density, cs, sigma_tot_e, sigma_tot_i, lo, hi);
    }
    for (auto &th : pool) th.join();
    return CUDAPIC_OK;
}
