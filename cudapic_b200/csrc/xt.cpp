// xt.cpp -- the XT diagnostics of a state on the host: eduPIC's
// normalisation, the derived currents and power absorption, and its files.
//
// Reference: norm_all_xt (C/eduPIC.cc:864-903), save_xt_1 / save_all_xt
// (:850-862, :905-918) and the <j E> power of check_and_save_info
// (:1011-1026).  With `cycles` the measured RF periods (measured steps /
// N_T), f1 = N_XT / (cycles N_T) and f2 = W / (A DX) / (cycles T / N_XT):
//   pot, efield, ne, ni      *= f1
//   ue = ue / counter_e,  je = -ue ne e,  meanee /= counter_e,  ioniz *= f2
//   ui = ui / counter_i,  ji =  ui ni e,  meanei /= counter_i
//   (each 0 where its counter is 0),  powere = je efield,  poweri = ji efield.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "internal.h"
#include "state_impl.h"

using namespace cudapic;

namespace cudapic {

// The eleven normalised quantities (CUDAPIC_XT_* order) from the raw
// accumulators; empty when the state has no XT diagnostics.
int xt_normalised(cudapic_state *s, std::vector<double> out[CUDAPIC_XT_QUANTITIES]) {
    if (!s->xt)
        return fail(CUDAPIC_ERR_NOT_SUPPORTED, "xt: no XT diagnostics (N_T not a multiple of 20, or never measured)");
    const cudapic_params &p = s->params;
    const size_t n_g = p.n_g, n_xt = s->n_xt, plane = n_g * n_xt;
    std::vector<double> raw((size_t)XT_RAW * plane);
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(raw.data(), s->xt, raw.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                             s->stream), "xt: download"));
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "xt: sync"));
    const double e_charge = 1.60217662e-19;
    const double cycles = (double)s->measure_steps / (double)p.n_t;
    const double period = 1.0 / p.frequency;
    const double dx = p.gap / (double)(p.n_g - 1);
    const double f1 = cycles > 0.0 ? (double)n_xt / (cycles * (double)p.n_t) : 0.0;
    const double f2 = cycles > 0.0 ? p.weight / (p.electrode_area * dx) / (cycles * (period / (double)n_xt)) : 0.0;
    for (int q = 0; q < CUDAPIC_XT_QUANTITIES; ++q) out[q].assign(plane, 0.0);
    auto R = [&](int q, size_t k) { return raw[(size_t)q * plane + k]; };
    for (size_t k = 0; k < plane; ++k) {
        const double ne = R(XT_NE, k) * f1, ni = R(XT_NI, k) * f1, ef = R(XT_EFIELD, k) * f1;
        out[CUDAPIC_XT_POT][k] = R(XT_POT, k) * f1;
        out[CUDAPIC_XT_EFIELD][k] = ef;
        out[CUDAPIC_XT_NE][k] = ne;
        out[CUDAPIC_XT_NI][k] = ni;
        const double ce = R(XT_COUNT_E, k), ci = R(XT_COUNT_I, k);
        if (ce > 0.0) {
            const double ue = R(XT_UE, k) / ce;
            out[CUDAPIC_XT_JE][k] = -ue * ne * e_charge;
            out[CUDAPIC_XT_MEANEE][k] = R(XT_MEANEE, k) / ce;
            out[CUDAPIC_XT_IONIZ][k] = R(XT_IONIZ, k) * f2;
        }
        if (ci > 0.0) {
            const double ui = R(XT_UI, k) / ci;
            out[CUDAPIC_XT_JI][k] = ui * ni * e_charge;
            out[CUDAPIC_XT_MEANEI][k] = R(XT_MEANEI, k) / ci;
        }
        out[CUDAPIC_XT_POWERE][k] = out[CUDAPIC_XT_JE][k] * ef;
        out[CUDAPIC_XT_POWERI][k] = out[CUDAPIC_XT_JI][k] * ef;
    }
    return CUDAPIC_OK;
}

// Space- and time-averaged electron and ion power absorption [W m^-3]
// (NaN without XT diagnostics).
int xt_power(cudapic_state *s, double *power_e, double *power_i) {
    *power_e = *power_i = NAN;
    if (!s->xt || s->measure_steps == 0) return CUDAPIC_OK;
    std::vector<double> q[CUDAPIC_XT_QUANTITIES];
    CUDAPIC_CHECK(xt_normalised(s, q));
    double pe = 0.0, pi = 0.0;
    for (size_t k = 0; k < q[CUDAPIC_XT_POWERE].size(); ++k) {
        pe += q[CUDAPIC_XT_POWERE][k];
        pi += q[CUDAPIC_XT_POWERI][k];
    }
    const double cells = (double)q[CUDAPIC_XT_POWERE].size();
    *power_e = pe / cells;
    *power_i = pi / cells;
    return CUDAPIC_OK;
}

}  // namespace cudapic

extern "C" int cudapic_state_xt_shape(const cudapic_state *s, uint32_t *n_g, uint32_t *n_xt) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_xt_shape: null state");
    if (n_g) *n_g = s->params.n_g;
    if (n_xt) *n_xt = s->xt ? s->n_xt : 0u;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_download_xt(cudapic_state *s, int quantity, double *out) {
    if (!s || !out) return fail(CUDAPIC_ERR_ARG, "state_download_xt: null pointer");
    if (quantity < 0 || quantity >= CUDAPIC_XT_QUANTITIES)
        return fail(CUDAPIC_ERR_ARG, "state_download_xt: bad quantity");
    DeviceGuard dg(s->device);
    std::vector<double> q[CUDAPIC_XT_QUANTITIES];
    CUDAPIC_CHECK(xt_normalised(s, q));
    std::copy(q[quantity].begin(), q[quantity].end(), out);
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_write_xt(cudapic_state *s, const char *directory) {
    if (!s || !directory) return fail(CUDAPIC_ERR_ARG, "state_write_xt: null pointer");
    DeviceGuard dg(s->device);
    std::vector<double> q[CUDAPIC_XT_QUANTITIES];
    CUDAPIC_CHECK(xt_normalised(s, q));
    static const char *names[CUDAPIC_XT_QUANTITIES] = {
        "pot_xt.dat", "efield_xt.dat", "ne_xt.dat", "ni_xt.dat", "je_xt.dat", "ji_xt.dat",
        "powere_xt.dat", "poweri_xt.dat", "meanee_xt.dat", "meanei_xt.dat", "ioniz_xt.dat"};
    const uint32_t n_g = s->params.n_g, n_xt = s->n_xt;
    for (int k = 0; k < CUDAPIC_XT_QUANTITIES; ++k) {
        const std::string path = std::string(directory) + "/" + names[k];
        FILE *f = std::fopen(path.c_str(), "w");
        if (!f) return fail(CUDAPIC_ERR_ARG, "state_write_xt: cannot open " + path);
        for (uint32_t i = 0; i < n_g; ++i) {
            for (uint32_t j = 0; j < n_xt; ++j) std::fprintf(f, "%e  ", q[k][(size_t)i * n_xt + j]);
            std::fprintf(f, "\n");
        }
        if (std::fclose(f) != 0) return fail(CUDAPIC_ERR_ARG, "state_write_xt: write failed: " + path);
    }
    return CUDAPIC_OK;
}
