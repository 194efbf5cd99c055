// report.cpp -- the simulation report's table-based numbers and the
// parameter-only stability precheck.
//
// Reference: max_electron_coll_freq / max_ion_coll_freq, C/eduPIC.cc:252-276
// (the largest collision frequency over the cross-section table, used by the
// accuracy conditions nu_max DT < 0.05 of check_and_save_info, :925-1030),
// and the Courant-Friedrichs-Levy energy 1/2 m (DX / DT_E)^2 (:974-977).
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "internal.h"

namespace cudapic {

namespace {
constexpr double kECharge = 1.60217662e-19;
constexpr double kEMass = 9.10938356e-31;
constexpr double kArMass = 6.63352090e-26;
constexpr double kDeCs = 0.001;  // eV per table entry
}  // namespace

void table_coll_freqs(const float *sigma_tot_e, const float *sigma_tot_i, double *max_e, double *max_i) {
    const double mu = 0.5 * kArMass;  // MU_ARAR
    double ne = 0.0, ni = 0.0;
    for (uint32_t k = 0; k < CUDAPIC_CS_RANGES; ++k) {
        const double e = (double)k * kDeCs;
        const double ve = std::sqrt(2.0 * e * kECharge / kEMass);
        const double gi = std::sqrt(2.0 * e * kECharge / mu);
        ne = std::max(ne, ve * (double)sigma_tot_e[k]);
        ni = std::max(ni, gi * (double)sigma_tot_i[k]);
    }
    *max_e = ne;
    *max_i = ni;
}

double cfl_max_energy(const cudapic_params &p) {
    const double dx = p.gap / (double)(p.n_g - 1);
    const double dt_e = 1.0 / (p.frequency * (double)p.n_t);
    const double v_max = dx / dt_e;
    return 0.5 * kEMass * v_max * v_max / kECharge;
}

}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_stability_precheck(const cudapic_params *p, cudapic_precheck *out) {
    CUDAPIC_REQUIRE(p && out, "stability_precheck: null pointer");
    cudapic_grid g;
    CUDAPIC_CHECK(cudapic_grid_from_params(p, &g));  // validates the parameters
    // The tables scale with the gas density: their maxima per unit density
    // are computed once per process.
    static std::mutex mu;
    static double unit_e = -1.0, unit_i = -1.0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (unit_e < 0.0) {
            std::vector<float> cs(5ull * CUDAPIC_CS_RANGES), se(CUDAPIC_CS_RANGES), si(CUDAPIC_CS_RANGES);
            CUDAPIC_CHECK(cudapic_cross_sections(1.0, cs.data(), se.data(), si.data()));
            table_coll_freqs(se.data(), si.data(), &unit_e, &unit_i);
        }
    }
    const double dt_e = 1.0 / (p->frequency * (double)p->n_t);
    out->max_e_coll_dt_e = unit_e * g.gas_density * dt_e;
    out->max_i_coll_dt_i = unit_i * g.gas_density * dt_e * (double)p->n_sub;
    out->cfl_max_energy = cfl_max_energy(*p);
    out->conditions_ok = out->max_e_coll_dt_e <= 0.05 && out->max_i_coll_dt_i <= 0.05;
    return CUDAPIC_OK;
}
