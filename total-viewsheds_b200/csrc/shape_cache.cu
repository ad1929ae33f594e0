// shape_cache.cu -- band shapes given as tables, and the reference's shape
// cache on disk.
//
// The reference computes one sector's band shape (DEM::calculate_axes +
// compile_band_data) or loads it from a cache (compute.rs:118-162):
//   <state_directory>/total-viewsheds/<dem_width>/band_deltas/<angle>.bin
//   <state_directory>/total-viewsheds/<dem_width>/distances/<angle>.bin
// raw native-endian i32 deltas and f32 distances, band_deltas_size of each
// (cache.rs:23-78).  A sector with both files is loaded, a sector without is
// computed and saved.  Here a loaded (or caller-given) shape is installed in
// the context: the shape stage then overwrites the computed tables of that
// sector with it (k_shape_tables) and derives the step tables from it, so
// every sweep path (surfaces, rings, FP64, MIXED64) runs on it.
//
// The reference keys the cache on the width alone, so two lines of sight on
// one width share files.  A table shorter than band_deltas_size is refused
// (the reference's kernel would index past it); a longer one contributes its
// first band_deltas_size entries, as the reference's kernel reads them.  A
// table that fills more steps than this geometry's band of sight is refused:
// it cannot come from this width and line of sight.  Rectangular DEMs (no
// counterpart in the reference) use the directory <width>x<height>.
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "tvs.h"
#include "tvs_internal.cuh"
#include "tvs_context.hpp"

namespace {

using tvs_host::fail_of;

#define TVS_CCUDA(ctx, expr)                                                              \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail_of(ctx, TVS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

std::string dem_directory(const tvs_context *c, const char *state_directory) {
    std::string d = std::string(state_directory) + "/total-viewsheds/" + std::to_string(c->g.width);
    if (c->g.height != c->g.width) d += "x" + std::to_string(c->g.height);
    return d;
}

std::string table_path(const std::string &dem_dir, const char *kind, uint32_t angle) {
    return dem_dir + "/" + kind + "/" + std::to_string(angle) + ".bin";
}

bool file_exists(const std::string &p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

// create_dir_all (cache.rs:44-48)
bool make_dirs(const std::string &path) {
    std::string cur;
    size_t i = 0;
    while (i <= path.size()) {
        size_t j = path.find('/', i);
        if (j == std::string::npos) j = path.size();
        cur = path.substr(0, j);
        if (!cur.empty() && mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) return false;
        i = j + 1;
    }
    struct stat st;
    return stat(path.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

template <typename T>
bool read_table(const std::string &p, std::vector<T> &out) {
    FILE *f = std::fopen(p.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0) { std::fclose(f); return false; }
    out.resize((size_t)n / sizeof(T));  // bytemuck::cast_slice needs whole elements
    const bool ok = (size_t)n % sizeof(T) == 0 &&
                    std::fread(out.data(), sizeof(T), out.size(), f) == out.size();
    std::fclose(f);
    return ok;
}

template <typename T>
bool write_table(const std::string &p, const T *v, size_t n) {
    FILE *f = std::fopen(p.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(v, sizeof(T), n, f) == n;
    return std::fclose(f) == 0 && ok;
}

int ensure_tables(tvs_context *c) {
    if (c->d_installed) return TVS_OK;
    const uint64_t bds = std::max<uint32_t>(c->g.band_deltas_size, 1);
    const uint64_t n = (uint64_t)tvs::kSectorSteps * bds;
    TVS_CCUDA(c, cudaMalloc(&c->d_tab_deltas, n * sizeof(int32_t)));
    TVS_CCUDA(c, cudaMalloc(&c->d_tab_dists, n * sizeof(float)));
    TVS_CCUDA(c, cudaMalloc(&c->d_installed, tvs::kSectorSteps));
    TVS_CCUDA(c, cudaMemsetAsync(c->d_installed, 0, tvs::kSectorSteps, c->stream));
    c->device_bytes += n * (sizeof(int32_t) + sizeof(float)) + tvs::kSectorSteps;
    return TVS_OK;
}

}  // namespace

extern "C" {

int tvs_set_band_shape(tvs_context *ctx, uint32_t angle, const int32_t *band_deltas,
                       const float *band_distances, uint64_t n) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (angle >= tvs::kSectorSteps || !band_deltas || !band_distances)
        return fail_of(ctx, TVS_ERR_INVALID_ARGUMENT, "angle >= 180 or a null table");
    const uint32_t bds = ctx->g.band_deltas_size;
    if (n < bds)
        return fail_of(ctx, TVS_ERR_SHAPE,
                       "band shape tables hold " + std::to_string(n) + " entries; this geometry reads " +
                           std::to_string(bds) + " (the reference's kernel would index past them)");
    uint32_t filled = 0;
    for (uint32_t i = 0; i < bds; i++) {
        uint32_t bits;
        std::memcpy(&bits, band_distances + i, sizeof bits);
        if (band_deltas[i] != 0 || bits != 0) filled = i + 1;
    }
    if (filled > ctx->g.band_steps_filled)
        return fail_of(ctx, TVS_ERR_SHAPE,
                       "band shape tables fill " + std::to_string(filled) + " steps; this width and "
                       "line of sight fill " + std::to_string(ctx->g.band_steps_filled) +
                       " (tables of another line of sight?)");
    TVS_CCUDA(ctx, cudaSetDevice(ctx->p.device));
    int rc = ensure_tables(ctx);
    if (rc) return rc;
    const uint64_t off = (uint64_t)angle * bds;
    const unsigned char one = 1;
    if (bds) {
        TVS_CCUDA(ctx, cudaMemcpyAsync(ctx->d_tab_deltas + off, band_deltas, bds * sizeof(int32_t),
                                       cudaMemcpyHostToDevice, ctx->stream));
        TVS_CCUDA(ctx, cudaMemcpyAsync(ctx->d_tab_dists + off, band_distances, bds * sizeof(float),
                                       cudaMemcpyHostToDevice, ctx->stream));
    }
    TVS_CCUDA(ctx, cudaMemcpyAsync(ctx->d_installed + angle, &one, 1, cudaMemcpyHostToDevice,
                                   ctx->stream));
    TVS_CCUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the host tables may go away
    if (!ctx->installed[angle]) tvs_host::drop_tvs_graph_of(ctx);  // one more shape launch
    ctx->installed[angle] = true;
    ctx->shape_ok[angle] = false;
    return TVS_OK;
}

int tvs_clear_band_shapes(tvs_context *ctx) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    for (bool &b : ctx->installed) b = false;
    for (bool &b : ctx->shape_ok) b = false;
    tvs_host::drop_tvs_graph_of(ctx);
    if (!ctx->d_installed) return TVS_OK;
    TVS_CCUDA(ctx, cudaSetDevice(ctx->p.device));
    TVS_CCUDA(ctx, cudaMemsetAsync(ctx->d_installed, 0, tvs::kSectorSteps, ctx->stream));
    TVS_CCUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TVS_OK;
}

int tvs_cache_load(tvs_context *ctx, const char *state_directory, uint32_t *sectors_loaded) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (!state_directory) return fail_of(ctx, TVS_ERR_INVALID_ARGUMENT, "null state directory");
    const std::string dir = dem_directory(ctx, state_directory);
    uint32_t loaded = 0;
    std::vector<int32_t> d;
    std::vector<float> x;
    for (uint32_t angle = 0; angle < tvs::kSectorSteps; angle++) {
        const std::string pd = table_path(dir, "band_deltas", angle);
        const std::string px = table_path(dir, "distances", angle);
        if (!file_exists(pd) || !file_exists(px)) continue;  // cache.rs:31 is_cache_exists
        if (!read_table(pd, d) || !read_table(px, x))
            return fail_of(ctx, TVS_ERR_INVALID_ARGUMENT, "cannot read the shape cache at " + pd);
        const uint64_t n = std::min<uint64_t>(d.size(), x.size());
        int rc = tvs_set_band_shape(ctx, angle, d.data(), x.data(), n);
        if (rc) {
            ctx->err = "shape cache " + pd + ": " + ctx->err;
            return rc;
        }
        loaded++;
    }
    if (sectors_loaded) *sectors_loaded = loaded;
    return TVS_OK;
}

int tvs_cache_save(tvs_context *ctx, const char *state_directory, int overwrite) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (!state_directory) return fail_of(ctx, TVS_ERR_INVALID_ARGUMENT, "null state directory");
    const std::string dir = dem_directory(ctx, state_directory);
    if (!make_dirs(dir + "/band_deltas") || !make_dirs(dir + "/distances"))
        return fail_of(ctx, TVS_ERR_INVALID_ARGUMENT, "cannot create the shape cache under " + dir);
    TVS_CCUDA(ctx, cudaSetDevice(ctx->p.device));
    int rc = tvs_host::enqueue_shape_of(ctx, 0, tvs::kSectorSteps);
    if (rc) return rc;
    const uint64_t bds = ctx->g.band_deltas_size;
    std::vector<int32_t> d(std::max<uint64_t>((uint64_t)tvs::kSectorSteps * bds, 1));
    std::vector<float> x(d.size());
    std::vector<tvs::ShapeHeader> h(tvs::kSectorSteps);
    if (bds) {
        TVS_CCUDA(ctx, cudaMemcpyAsync(d.data(), ctx->d_deltas, tvs::kSectorSteps * bds * sizeof(int32_t),
                                       cudaMemcpyDeviceToHost, ctx->stream));
        TVS_CCUDA(ctx, cudaMemcpyAsync(x.data(), ctx->d_dists, tvs::kSectorSteps * bds * sizeof(float),
                                       cudaMemcpyDeviceToHost, ctx->stream));
    }
    TVS_CCUDA(ctx, cudaMemcpyAsync(h.data(), ctx->d_hdr, tvs::kSectorSteps * sizeof(tvs::ShapeHeader),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    TVS_CCUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (uint32_t angle = 0; angle < tvs::kSectorSteps; angle++) {
        // the reference saves a shape whose bands leave the DEM too (its kernel
        // fails later); any other shape-stage failure has no tables to save
        if (h[angle].status != TVS_OK && h[angle].status != TVS_ERR_PATH_OUT_OF_DEM)
            return tvs_host::header_status_of(ctx, angle, 1);
        const std::string pd = table_path(dir, "band_deltas", angle);
        const std::string px = table_path(dir, "distances", angle);
        if (!overwrite && file_exists(pd) && file_exists(px)) continue;
        if (!write_table(pd, d.data() + angle * bds, bds) || !write_table(px, x.data() + angle * bds, bds))
            return fail_of(ctx, TVS_ERR_INVALID_ARGUMENT, "cannot write the shape cache at " + pd);
    }
    return TVS_OK;
}

}  // extern "C"
