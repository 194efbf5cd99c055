// checkpoint.cpp -- eduPIC's particle checkpoint file (picdata.bin).
//
// Reference: save_particle_data / load_particle_data, C/eduPIC.cc:726-781.
// The file is a sequence of doubles:
//   Time [s], cycles_done, N_e, x_e[N_e], vx_e[N_e], vy_e[N_e], vz_e[N_e],
//   N_i, x_i[N_i], vx_i[N_i], vy_i[N_i], vz_i[N_i]
// (native byte order, as eduPIC writes it).  Particles here are f32: writing
// widens exactly, reading rounds each double to the nearest f32.
//
// The RNG sidecar (<path>.rng) is this library's own: the xoshiro128+ planes
// of both species over every slot, so that a resumed run continues the same
// streams.  Layout: the 8 bytes "CPICRNG1", u32 capacity, u32 0, then for
// electrons and ions the planes rng0..rng3, capacity u32 each.
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

namespace {

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

bool write_doubles(FILE *f, const double *p, size_t n) { return std::fwrite(p, sizeof(double), n, f) == n; }
bool read_doubles(FILE *f, double *p, size_t n) { return std::fread(p, sizeof(double), n, f) == n; }

int write_species(FILE *f, const float *const planes[4], uint32_t n) {
    const double count = (double)n;
    if (!write_doubles(f, &count, 1)) return cudapic::fail(CUDAPIC_ERR_ARG, "picdata: write failed");
    std::vector<double> buf(n);
    for (int a = 0; a < 4; ++a) {
        for (uint32_t k = 0; k < n; ++k) buf[k] = (double)planes[a][k];
        if (n && !write_doubles(f, buf.data(), n)) return cudapic::fail(CUDAPIC_ERR_ARG, "picdata: write failed");
    }
    return CUDAPIC_OK;
}

// Reads a count; a count that is not a non-negative integer below 2^32 is a malformed file.
int read_count(FILE *f, uint32_t *n) {
    double d = 0.0;
    if (!read_doubles(f, &d, 1)) return cudapic::fail(CUDAPIC_ERR_ARG, "picdata: truncated file");
    if (!(d >= 0.0 && d < 4294967296.0) || d != (double)(uint64_t)d)
        return cudapic::fail(CUDAPIC_ERR_ARG, "picdata: bad particle count");
    *n = (uint32_t)d;
    return CUDAPIC_OK;
}

int read_species(FILE *f, float *const planes[4], uint32_t n) {
    std::vector<double> buf(n);
    for (int a = 0; a < 4; ++a) {
        if (n && !read_doubles(f, buf.data(), n)) return cudapic::fail(CUDAPIC_ERR_ARG, "picdata: truncated file");
        for (uint32_t k = 0; k < n; ++k) planes[a][k] = (float)buf[k];
    }
    return CUDAPIC_OK;
}

}  // namespace

using namespace cudapic;

extern "C" int cudapic_picdata_write(const char *path, double time, uint32_t cycles_done, const float *const e[4],
                                     uint32_t n_e, const float *const i[4], uint32_t n_i) {
    CUDAPIC_REQUIRE(path && e && i, "picdata_write: null pointer");
    for (int a = 0; a < 4; ++a) CUDAPIC_REQUIRE((e[a] || !n_e) && (i[a] || !n_i), "picdata_write: null plane");
    File file(path, "wb");
    if (!file.f) return fail(CUDAPIC_ERR_ARG, std::string("picdata_write: cannot open ") + path);
    const double head[2] = {time, (double)cycles_done};
    if (!write_doubles(file.f, head, 2)) return fail(CUDAPIC_ERR_ARG, "picdata: write failed");
    CUDAPIC_CHECK(write_species(file.f, e, n_e));
    CUDAPIC_CHECK(write_species(file.f, i, n_i));
    return CUDAPIC_OK;
}

extern "C" int cudapic_picdata_read_header(const char *path, double *time, uint32_t *cycles_done, uint32_t *n_e,
                                           uint32_t *n_i) {
    CUDAPIC_REQUIRE(path, "picdata_read_header: null path");
    File file(path, "rb");
    if (!file.f) return fail(CUDAPIC_ERR_ARG, std::string("picdata_read_header: cannot open ") + path);
    double head[2];
    if (!read_doubles(file.f, head, 2)) return fail(CUDAPIC_ERR_ARG, "picdata: truncated file");
    uint32_t ne = 0, ni = 0;
    CUDAPIC_CHECK(read_count(file.f, &ne));
    if (std::fseek(file.f, (long)(4ull * ne * sizeof(double)), SEEK_CUR) != 0)
        return fail(CUDAPIC_ERR_ARG, "picdata: truncated file");
    CUDAPIC_CHECK(read_count(file.f, &ni));
    // eduPIC truncates the stored cycle count with int() (C/eduPIC.cc:767);
    // a value that is no count at all (negative, NaN, 2^32 or more) is a malformed file
    if (!(head[1] >= 0.0 && head[1] < 4294967296.0)) return fail(CUDAPIC_ERR_ARG, "picdata: bad cycle count");
    if (time) *time = head[0];
    if (cycles_done) *cycles_done = (uint32_t)head[1];
    if (n_e) *n_e = ne;
    if (n_i) *n_i = ni;
    return CUDAPIC_OK;
}

extern "C" int cudapic_picdata_read(const char *path, float *const e[4], uint32_t max_e, float *const i[4],
                                    uint32_t max_i) {
    CUDAPIC_REQUIRE(path && e && i, "picdata_read: null pointer");
    File file(path, "rb");
    if (!file.f) return fail(CUDAPIC_ERR_ARG, std::string("picdata_read: cannot open ") + path);
    double head[2];
    if (!read_doubles(file.f, head, 2)) return fail(CUDAPIC_ERR_ARG, "picdata: truncated file");
    uint32_t ne = 0, ni = 0;
    CUDAPIC_CHECK(read_count(file.f, &ne));
    if (ne > max_e) return fail(CUDAPIC_ERR_CAPACITY, "picdata_read: more electrons than max_e");
    for (int a = 0; a < 4; ++a) CUDAPIC_REQUIRE(e[a] || !ne, "picdata_read: null plane");
    CUDAPIC_CHECK(read_species(file.f, e, ne));
    CUDAPIC_CHECK(read_count(file.f, &ni));
    if (ni > max_i) return fail(CUDAPIC_ERR_CAPACITY, "picdata_read: more ions than max_i");
    for (int a = 0; a < 4; ++a) CUDAPIC_REQUIRE(i[a] || !ni, "picdata_read: null plane");
    return read_species(file.f, i, ni);
}

namespace cudapic {

static const char kRngMagic[8] = {'C', 'P', 'I', 'C', 'R', 'N', 'G', '1'};

int rng_sidecar_write(const char *path, uint32_t capacity, const std::vector<uint32_t> planes[2][4]) {
    const std::string p = std::string(path) + ".rng";
    File file(p.c_str(), "wb");
    if (!file.f) return fail(CUDAPIC_ERR_ARG, "state_save: cannot open " + p);
    const uint32_t head[2] = {capacity, 0u};
    bool ok = std::fwrite(kRngMagic, 1, 8, file.f) == 8 && std::fwrite(head, sizeof(uint32_t), 2, file.f) == 2;
    for (int sp = 0; sp < 2 && ok; ++sp)
        for (int k = 0; k < 4 && ok; ++k)
            ok = std::fwrite(planes[sp][k].data(), sizeof(uint32_t), capacity, file.f) == capacity;
    return ok ? CUDAPIC_OK : fail(CUDAPIC_ERR_ARG, "state_save: write failed: " + p);
}

// CUDAPIC_ERR_NOT_SUPPORTED (nothing recorded) when the sidecar does not exist.
int rng_sidecar_read(const char *path, uint32_t capacity, std::vector<uint32_t> planes[2][4]) {
    const std::string p = std::string(path) + ".rng";
    File file(p.c_str(), "rb");
    if (!file.f) return CUDAPIC_ERR_NOT_SUPPORTED;
    char magic[8];
    uint32_t head[2];
    if (std::fread(magic, 1, 8, file.f) != 8 || std::memcmp(magic, kRngMagic, 8) != 0 ||
        std::fread(head, sizeof(uint32_t), 2, file.f) != 2)
        return fail(CUDAPIC_ERR_ARG, "state_load: not an RNG sidecar: " + p);
    if (head[0] != capacity) return fail(CUDAPIC_ERR_ARG, "state_load: RNG sidecar written for another capacity");
    for (int sp = 0; sp < 2; ++sp)
        for (int k = 0; k < 4; ++k) {
            planes[sp][k].resize(capacity);
            if (std::fread(planes[sp][k].data(), sizeof(uint32_t), capacity, file.f) != capacity)
                return fail(CUDAPIC_ERR_ARG, "state_load: truncated RNG sidecar");
        }
    return CUDAPIC_OK;
}

}  // namespace cudapic
