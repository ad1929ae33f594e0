// batch.cu -- many DEM tiles, all 180 sectors each, per CUDA-graph replay.
//
// A batch holds one context per DEM (its elevations, sector tables and
// surfaces) and replays one captured graph per run:
//   * the surfaces of every DEM are zeroed,
//   * one shape launch computes every (DEM, sector) table (one CTA each),
//   * one persistent sweep takes (sector, DEM, tile) items from a single
//     queue, so uneven and rectangular DEMs share the GPU without a tail per
//     DEM (sweep_queue.cu).
// The sweep configuration (points of view per thread, tile shape, packed
// arithmetic) comes from tvs_batch_autotune, which times the candidates on a
// few sectors of the batch itself.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "tvs.h"
#include "tvs_context.hpp"
#include "tvs_internal.cuh"

struct tvs_batch {
    int device = 0;
    uint32_t precision = 0;
    cudaStream_t stream = nullptr;
    std::vector<tvs_context *> dems;
    tvs::ShapeArgs *d_shape = nullptr;
    tvs::QueueDem *d_dems = nullptr;
    uint32_t *d_queue = nullptr;
    uint32_t *d_done = nullptr;
    uint32_t done_cap = 0;
    int32_t *d_error = nullptr;
    unsigned long long *d_rechecks = nullptr;
    uint32_t max_step_cap = 0;
    uint32_t tiles_per_sector = 0;
    tvs::QueueConfig cfg{0, 0, 0, 0, 0};
    bool dems_uploaded = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string err;
    uint64_t device_bytes = 0;
};

namespace {

int bfail(tvs_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg; else tvs_set_create_error(msg);
    return code;
}

#define TVS_BCUDA(b, expr)                                                                   \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess) return bfail(b, TVS_ERR_CUDA, std::string(#expr ": ") +       \
                                                                   cudaGetErrorString(e_));   \
    } while (0)

void drop_graph(tvs_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// The DEM descriptors tiled for the batch's configuration.
int upload_dems(tvs_batch *b) {
    if (b->dems_uploaded) return TVS_OK;
    std::vector<tvs::QueueDem> d(b->dems.size());
    for (size_t i = 0; i < d.size(); i++) d[i] = tvs_host::queue_dem_of(b->dems[i]);
    uint32_t done_total = 0;
    tvs::queue_tile(d.data(), (uint32_t)d.size(), b->cfg, &b->tiles_per_sector, &done_total);
    if (done_total > b->done_cap) return bfail(b, TVS_ERR_CAPACITY, "batch tile counters");
    TVS_BCUDA(b, cudaMemcpy(b->d_dems, d.data(), d.size() * sizeof(tvs::QueueDem),
                            cudaMemcpyHostToDevice));
    b->dems_uploaded = true;
    return TVS_OK;
}

tvs::QueueArgs queue_args(const tvs_batch *b, uint32_t first, uint32_t count) {
    tvs::QueueArgs q{};
    q.dems = b->d_dems;
    q.n_dems = (uint32_t)b->dems.size();
    q.first_sector = first;
    q.n_sectors = count;
    q.tiles_per_sector = b->tiles_per_sector;
    q.max_step_cap = b->max_step_cap;
    q.queue = b->d_queue;
    q.done = b->d_done;
    q.done_total = b->tiles_per_sector;
    q.done_cap = b->done_cap;
    q.error = b->d_error;
    q.spin_limit = tvs::kDefaultSpinLimit;
    q.held_tile = 0xFFFFFFFFu;
    q.rechecks = b->d_rechecks;
    return q;
}

// Zero every DEM's surfaces, compute every table, sweep sectors [0, count).
int enqueue_run(tvs_batch *b, uint32_t count) {
    for (tvs_context *c : b->dems) {
        const uint64_t n = std::max<uint64_t>(c->g.computable_points_count, 1);
        TVS_BCUDA(b, cudaMemsetAsync(c->d_cum, 0, n * sizeof(float), b->stream));
        TVS_BCUDA(b, cudaMemsetAsync(c->d_total, 0, n * sizeof(float), b->stream));
        if (c->d_cum64) TVS_BCUDA(b, cudaMemsetAsync(c->d_cum64, 0, n * sizeof(double), b->stream));
    }
    TVS_BCUDA(b, tvs::launch_shape_batch(b->d_shape, (uint32_t)b->dems.size(), tvs::kSectorSteps,
                                         b->stream));
    // the quad layout needs every DEM's row-interleaved copies, else its tiling
    // runs from the plain DEMs
    tvs::QueueConfig cfg = b->cfg;
    if (cfg.layout == tvs::kQuadLayout)
        for (const tvs_context *c : b->dems)
            if (!c->d_quad) cfg.layout = tvs::kQuadFallback;
    TVS_BCUDA(b, tvs::launch_sweep_queue(queue_args(b, 0, count), (int)b->precision, cfg,
                                         b->stream));
    return TVS_OK;
}

}  // namespace

extern "C" {

int tvs_batch_create(const tvs_params *params, const float *const *elevations, uint32_t n_dems,
                     tvs_batch **out) {
    if (!params || !elevations || !out || n_dems == 0)
        return bfail(nullptr, TVS_ERR_INVALID_ARGUMENT, "null argument or empty batch");
    *out = nullptr;
    for (uint32_t i = 1; i < n_dems; i++)
        if (params[i].device != params[0].device || params[i].precision != params[0].precision)
            return bfail(nullptr, TVS_ERR_INVALID_ARGUMENT,
                         "every DEM of a batch needs the same device and precision");
    if (params[0].sweep_kernel != TVS_SWEEP_ENGINE)
        return bfail(nullptr, TVS_ERR_INVALID_ARGUMENT, "batches use the engine sweep");
    tvs_batch *b = new tvs_batch();
    b->device = params[0].device;
    b->precision = params[0].precision;
    auto bail = [&](int code) {
        tvs_batch_destroy(b);
        return code;
    };
    for (uint32_t i = 0; i < n_dems; i++) {
        tvs_context *c = nullptr;
        tvs_params p = params[i];
        p.tvs_row_begin = p.tvs_row_end = 0;
        const uint64_t n = (uint64_t)p.width * p.height;
        int rc = tvs_create(&p, elevations[i], n, &c);
        if (rc) {
            std::string m = std::string("DEM ") + std::to_string(i) + ": " + tvs_last_error(nullptr);
            bail(rc);
            return bfail(nullptr, rc, m);
        }
        b->dems.push_back(c);
        b->device_bytes += tvs_device_bytes(c);
        b->max_step_cap = std::max(b->max_step_cap, c->step_cap);
        b->done_cap += c->done_cap;
    }
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    std::vector<tvs::ShapeArgs> sa(n_dems);
    for (uint32_t i = 0; i < n_dems; i++) sa[i] = tvs_host::shape_args_of(b->dems[i], 0);
    struct { void **p; size_t bytes; } allocs[] = {
        {(void **)&b->d_shape, n_dems * sizeof(tvs::ShapeArgs)},
        {(void **)&b->d_dems, n_dems * sizeof(tvs::QueueDem)},
        {(void **)&b->d_queue, sizeof(uint32_t)},
        {(void **)&b->d_done, (size_t)b->done_cap * sizeof(uint32_t)},
        {(void **)&b->d_error, sizeof(int32_t)},
        {(void **)&b->d_rechecks, sizeof(unsigned long long)},
    };
    for (auto &a : allocs) {
        if (e == cudaSuccess) e = cudaMalloc(a.p, a.bytes);
        if (e == cudaSuccess) b->device_bytes += a.bytes;
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_shape, sa.data(), n_dems * sizeof(tvs::ShapeArgs), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->d_error, 0, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(b->d_rechecks, 0, sizeof(unsigned long long));
    // configure the shape kernel (a function attribute) outside any capture
    if (e == cudaSuccess) e = tvs::launch_shape_batch(b->d_shape, 0, tvs::kSectorSteps, b->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        std::string m = std::string("batch set-up: ") + cudaGetErrorString(e);
        bail(e == cudaErrorMemoryAllocation ? TVS_ERR_OUT_OF_MEMORY : TVS_ERR_CUDA);
        return bfail(nullptr, e == cudaErrorMemoryAllocation ? TVS_ERR_OUT_OF_MEMORY : TVS_ERR_CUDA, m);
    }
    b->cfg = tvs::default_queue_config((int)b->precision);
    int rc = upload_dems(b);
    if (rc) {
        std::string m = b->err;
        bail(rc);
        return bfail(nullptr, rc, m);
    }
    *out = b;
    return TVS_OK;
}

void tvs_batch_destroy(tvs_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    void *ptrs[] = {b->d_shape, b->d_dems, b->d_queue, b->d_done, b->d_error, b->d_rechecks};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (tvs_context *c : b->dems) tvs_destroy(c);
    delete b;
}

const char *tvs_batch_last_error(const tvs_batch *b) {
    return b ? b->err.c_str() : tvs_last_error(nullptr);
}

uint32_t tvs_batch_size(const tvs_batch *b) { return b ? (uint32_t)b->dems.size() : 0; }

int tvs_batch_geometry(const tvs_batch *b, uint32_t dem, tvs_geometry *out) {
    if (!b || !out || dem >= b->dems.size()) return TVS_ERR_INVALID_ARGUMENT;
    return tvs_get_geometry(b->dems[dem], out);
}

int tvs_batch_set_sweep_config(tvs_batch *b, const tvs_sweep_config *cfg) {
    if (!b || !cfg) return TVS_ERR_INVALID_ARGUMENT;
    tvs::QueueConfig c{cfg->points_x, cfg->points_y, cfg->packed != 0, cfg->prefetch != 0, cfg->layout};
    if (!tvs::queue_config_valid(c))
        return bfail(b, TVS_ERR_INVALID_ARGUMENT, "unsupported points-per-thread shape");
    if (c.layout != 0 && b->precision == TVS_PRECISION_FP64)
        return bfail(b, TVS_ERR_INVALID_ARGUMENT, "sweep layouts 1-9 are not available for FP64");
    if (c.layout == 0 && b->precision == TVS_PRECISION_FP32)
        return bfail(b, TVS_ERR_INVALID_ARGUMENT, "the FP32 form runs on sweep layouts 1-9 only");
    if (c.px != b->cfg.px || c.py != b->cfg.py || c.packed != b->cfg.packed ||
        c.prefetch != b->cfg.prefetch || c.layout != b->cfg.layout) {
        b->cfg = c;
        b->dems_uploaded = false;
        drop_graph(b);
    }
    return upload_dems(b);
}

int tvs_batch_get_sweep_config(const tvs_batch *b, tvs_sweep_config *cfg) {
    if (!b || !cfg) return TVS_ERR_INVALID_ARGUMENT;
    cfg->points_x = b->cfg.px;
    cfg->points_y = b->cfg.py;
    cfg->packed = b->cfg.packed;
    cfg->prefetch = b->cfg.prefetch;
    cfg->layout = b->cfg.layout;
    return TVS_OK;
}

int tvs_batch_autotune(tvs_batch *b, uint32_t sample_sectors, tvs_sweep_config *chosen) {
    if (!b) return TVS_ERR_INVALID_ARGUMENT;
    if (sample_sectors == 0 || sample_sectors > tvs::kSectorSteps)
        return bfail(b, TVS_ERR_INVALID_ARGUMENT, "sample_sectors must be in [1, 180]");
    TVS_BCUDA(b, cudaSetDevice(b->device));
    const bool exact = b->precision == TVS_PRECISION_EXACT32;
    const bool f64 = b->precision == TVS_PRECISION_FP64;
    const bool fp32 = b->precision == TVS_PRECISION_FP32;
    const tvs::QueueConfig cands[] = {{1, 1, 0, 0, 0}, {2, 1, 0, 0, 0}, {4, 1, 0, 0, 0},
                                      {2, 2, 0, 0, 0}, {2, 1, 1, 0, 0}, {4, 1, 1, 0, 0},
                                      {1, 1, 0, 1, 0}, {2, 1, 0, 1, 0}, {4, 1, 0, 1, 0},
                                      {2, 2, 0, 1, 0}, {4, 1, 0, 0, 1}, {4, 1, 0, 0, 2},
                                      {4, 1, 0, 0, 3}, {4, 1, 0, 0, 4}, {4, 1, 0, 0, 5},
                                      {4, 1, 0, 0, 6}, {4, 1, 0, 0, 7}, {4, 1, 0, 0, 8},
                                      {4, 1, 0, 0, 9}};
    cudaEvent_t t0, t1;
    TVS_BCUDA(b, cudaEventCreate(&t0));
    TVS_BCUDA(b, cudaEventCreate(&t1));
    float best = 1e30f;
    tvs::QueueConfig best_cfg = b->cfg;
    int rc = TVS_OK;
    for (const tvs::QueueConfig &c : cands) {
        if ((c.packed && !exact) || (c.layout != 0 && f64) || (c.layout == 0 && fp32)) continue;
        tvs_sweep_config sc{c.px, c.py, c.packed, c.prefetch, c.layout};
        if ((rc = tvs_batch_set_sweep_config(b, &sc))) break;
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && rc == TVS_OK; rep++) {  // the first run warms up
            cudaEventRecord(t0, b->stream);
            rc = enqueue_run(b, sample_sectors);
            cudaEventRecord(t1, b->stream);
            if (rc == TVS_OK && cudaEventSynchronize(t1) != cudaSuccess)
                rc = bfail(b, TVS_ERR_CUDA, "autotune run failed");
            if (rc == TVS_OK) cudaEventElapsedTime(&ms, t0, t1);
        }
        if (rc) break;
        if (ms < best) {
            best = ms;
            best_cfg = c;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    tvs_sweep_config sc{best_cfg.px, best_cfg.py, best_cfg.packed, best_cfg.prefetch, best_cfg.layout};
    rc = tvs_batch_set_sweep_config(b, &sc);
    if (rc == TVS_OK && chosen) *chosen = sc;
    return rc;
}

int tvs_batch_run(tvs_batch *b) {
    if (!b) return TVS_ERR_INVALID_ARGUMENT;
    TVS_BCUDA(b, cudaSetDevice(b->device));
    int rc = upload_dems(b);
    if (rc) return rc;
    if (!b->exec) {
        TVS_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_run(b, tvs::kSectorSteps);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return bfail(b, TVS_ERR_CUDA, std::string("graph capture: ") +
                                                                cudaGetErrorString(e));
        b->graph = g;
        TVS_BCUDA(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    TVS_BCUDA(b, cudaGraphLaunch(b->exec, b->stream));
    return TVS_OK;
}

int tvs_batch_finish(tvs_batch *b) {
    if (!b) return TVS_ERR_INVALID_ARGUMENT;
    TVS_BCUDA(b, cudaSetDevice(b->device));
    TVS_BCUDA(b, cudaStreamSynchronize(b->stream));
    for (size_t i = 0; i < b->dems.size(); i++) {
        int rc = tvs_host::header_status_of(b->dems[i], 0, tvs::kSectorSteps);
        if (rc) return bfail(b, rc, "DEM " + std::to_string(i) + ": " + tvs_last_error(b->dems[i]));
    }
    int32_t err = 0;
    TVS_BCUDA(b, cudaMemcpy(&err, b->d_error, sizeof err, cudaMemcpyDeviceToHost));
    if (err) {
        TVS_BCUDA(b, cudaMemset(b->d_error, 0, sizeof err));
        return bfail(b, err, "batch sweep: a tile's dependency wait gave up (iteration limit)");
    }
    return TVS_OK;
}

int tvs_batch_read(tvs_batch *b, uint32_t dem, float *cumulative_out, float *total_out) {
    if (!b || dem >= b->dems.size()) return TVS_ERR_INVALID_ARGUMENT;
    tvs_context *c = b->dems[dem];
    const uint64_t n = c->g.computable_points_count;
    TVS_BCUDA(b, cudaSetDevice(b->device));
    TVS_BCUDA(b, cudaStreamSynchronize(b->stream));
    if (cumulative_out && n)
        TVS_BCUDA(b, cudaMemcpy(cumulative_out, c->d_cum, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (total_out && n)
        TVS_BCUDA(b, cudaMemcpy(total_out, c->d_total, n * sizeof(float), cudaMemcpyDeviceToHost));
    return TVS_OK;
}

void *tvs_batch_stream(const tvs_batch *b) { return b ? (void *)b->stream : nullptr; }

uint64_t tvs_batch_device_bytes(const tvs_batch *b) { return b ? b->device_bytes : 0; }

}  // extern "C"
