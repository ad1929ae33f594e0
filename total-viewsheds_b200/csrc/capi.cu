// capi.cu -- the extern "C" boundary (include/tvs.h) and the per-context
// orchestration of the shape and sweep stages.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "tvs.h"
#include "tvs_internal.cuh"

#include "tvs_context.hpp"

namespace {

thread_local std::string g_create_error;

constexpr double kRadsPerDeg = 3.14159265358979323846 / 180.0;  // Rust f64::to_radians
constexpr double kSqrt2 = 1.41421356237309504880;               // core::f64::consts::SQRT_2
constexpr uint32_t kSpillCap = 1u << 22;

int fail(tvs_context *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg; else g_create_error = msg;
    return code;
}

int cuda_fail(tvs_context *ctx, cudaError_t e, const char *what) {
    return fail(ctx, TVS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define TVS_CUDA(ctx, expr)                                   \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #expr); \
    } while (0)

// Rust `f32 as u32` (saturating, NaN -> 0).
uint32_t f32_as_u32(float v) {
    if (!(v > 0.0f)) return 0;
    if (v >= 4294967296.0f) return UINT32_MAX;
    return (uint32_t)v;
}

// dem.rs:106-115 along one axis (the test is separable for a rectangle).
uint32_t computable_along(uint32_t extent, float scale, uint32_t los_m) {
    const float lower = (float)los_m;
    const float upper = ((float)(extent - 1) * scale) - lower;
    uint32_t n = 0;
    for (uint32_t i = 0; i < extent; i++) {
        const float v = (float)i * scale;
        if (v >= lower && v <= upper) n++;
    }
    return n;
}

uint64_t isqrt_u64(uint64_t n) {
    uint64_t r = (uint64_t)std::sqrt((double)n);
    while (r * r > n) r--;
    while ((r + 1) * (r + 1) <= n) r++;
    return r;
}

// DEM::new (dem.rs:44-72), Compute::new (compute.rs:34-47) and the index
// ranges compile_band_data relies on (band_of_sight.rs:95-165).  Returns an
// error where the reference bails or panics.
int derive_geometry(const tvs_params *p, tvs_geometry *g, std::string *msg) {
    std::memset(g, 0, sizeof(*g));
    if (!p || p->width == 0 || p->height == 0) {
        *msg = "width and height must be positive";
        return TVS_ERR_INVALID_ARGUMENT;
    }
    if (!(p->scale > 0.0f) || !std::isfinite(p->scale)) {
        *msg = "scale must be a positive finite number of metres";
        return TVS_ERR_INVALID_ARGUMENT;
    }
    g->width = p->width;
    g->height = p->height;
    g->size = (uint64_t)p->width * p->height;
    if (g->size >= (1ull << 31)) {
        *msg = "DEM ids must fit in i32 (band_of_sight.rs:160)";
        return TVS_ERR_INVALID_ARGUMENT;
    }
    g->max_los_as_points = f32_as_u32((float)p->max_line_of_sight / p->scale);
    const uint32_t shorter = std::min(p->width, p->height);
    if (g->max_los_as_points > shorter / 2) {
        char b[256];
        std::snprintf(b, sizeof b,
                      "The maximum line of sight (%um) is longer than the maximum distance "
                      "that any point can completely see (%gm).",
                      p->max_line_of_sight, (double)(shorter / 2) * (double)p->scale);
        *msg = b;
        return TVS_ERR_LOS_TOO_LONG;
    }
    g->band_size = g->max_los_as_points + 1;
    g->band_deltas_size = g->band_size - 1;
    const uint32_t nx = computable_along(p->width, p->scale, p->max_line_of_sight);
    const uint32_t ny = computable_along(p->height, p->scale, p->max_line_of_sight);
    g->computable_points_count = (uint64_t)nx * ny;
    if (p->width == p->height) {
        g->tvs_width = (uint32_t)isqrt_u64(g->computable_points_count);
        g->tvs_height = g->tvs_width;
    } else {
        g->tvs_width = nx;
        g->tvs_height = ny;
    }
    g->total_bands = 2 * g->computable_points_count;
    const float band_length_in_km = (float)p->max_line_of_sight / 1000.0f;
    g->reserved_rings_per_band = f32_as_u32(band_length_in_km * p->rings_per_km);
    g->ring_slots_per_sector = g->total_bands * g->reserved_rings_per_band;
    const uint64_t bs = (uint64_t)((double)(g->band_size * 2) * kSqrt2);
    g->band_samples = (uint32_t)bs;
    const uint64_t middle = bs / 2, end = 2ull * g->band_size;
    // the shape is built on the central min(W, H) square (the whole DEM when square)
    const uint64_t win = (uint64_t)shorter * shorter;
    if (bs / 2 > win / 2 || win / 2 - bs / 2 + bs > win || end >= bs ||
        end - middle > g->band_deltas_size) {
        *msg = "line of sight too short for the band-of-sight shape (band_of_sight.rs:103-165 "
               "index out of bounds)";
        return TVS_ERR_SHAPE;
    }
    g->band_steps_filled = (uint32_t)(end - middle);
    if (bs > tvs::kWindowCap ||
        (uint64_t)(g->band_deltas_size + 2) * 8 + (uint64_t)g->band_deltas_size * 4 >
            (uint64_t)tvs::kCandidateCap * 8) {
        *msg = "band_samples exceeds the shape stage's shared-memory capacity";
        return TVS_ERR_CAPACITY;
    }
    return TVS_OK;
}

// The captured whole-TVS graph depends on the sweep configuration, the
// installed shapes, the wait settings and the counters: any change drops it.
void drop_tvs_graph(tvs_context *c) {
    if (c->tvs_exec) cudaGraphExecDestroy(c->tvs_exec);
    if (c->tvs_graph) cudaGraphDestroy(c->tvs_graph);
    c->tvs_exec = nullptr;
    c->tvs_graph = nullptr;
}

void free_all(tvs_context *c) {
    void *ptrs[] = {c->d_elev, c->d_cum, c->d_total, c->d_cum64, c->d_trig, c->d_hdr,
                    c->d_steps, c->d_offs, c->d_dtab, c->d_queue, c->d_done, c->d_error, c->d_hmax,
                    c->d_rechecks, c->d_qdem,
                    c->d_deltas, c->d_dists, c->d_rings, c->d_spill, c->d_counters, c->d_sf,
                    c->d_sb, c->d_tab_deltas, c->d_tab_dists, c->d_installed,
                    c->d_rc_blocks, c->d_rc_offsets, c->d_rc_ids, c->d_bmax, c->d_qdem_rings,
                    c->d_diag, c->d_quad};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    drop_tvs_graph(c);
    for (cudaEvent_t ev : {c->ev_begin, c->ev_shaped, c->ev_swept})
        if (ev) cudaEventDestroy(ev);
    if (c->stream) cudaStreamDestroy(c->stream);
}

tvs::ShapeArgs shape_args(tvs_context *c, uint32_t first_slot) {
    tvs::ShapeArgs a{};
    a.width = c->g.width;
    a.height = c->g.height;
    a.size = c->g.size;
    a.win = std::min(c->g.width, c->g.height);
    a.x0 = (c->g.width - a.win) / 2;
    a.y0 = (c->g.height - a.win) / 2;
    a.band_size = c->g.band_size;
    a.band_deltas_size = c->g.band_deltas_size;
    a.band_samples = c->g.band_samples;
    a.first_angle = first_slot;
    a.step_cap = c->step_cap;
    a.pov_min = c->pov_min;
    a.pov_max = c->pov_max;
    a.trig = c->d_trig + first_slot;
    a.hdr = c->d_hdr + first_slot;
    a.steps = c->d_steps + (uint64_t)first_slot * c->step_cap;
    a.offs = c->d_offs + (uint64_t)first_slot * c->step_cap;
    a.dtab = c->d_dtab + (uint64_t)first_slot * c->step_cap;
    a.deltas = c->d_deltas + (uint64_t)first_slot * c->g.band_deltas_size;
    a.dists = c->d_dists + (uint64_t)first_slot * c->g.band_deltas_size;
    return a;
}

tvs::SweepArgs sweep_args(tvs_context *c, uint32_t first, uint32_t count) {
    tvs::SweepArgs a{};
    a.elev = c->d_elev;
    a.width = c->g.width;
    a.tvs_width = c->g.tvs_width;
    a.row_begin = c->row_begin;
    a.row_end = c->row_end;
    a.los = c->g.max_los_as_points;
    a.observer_height = c->p.observer_height;
    a.n_sectors = count;
    a.step_cap = c->step_cap;
    a.hdr = c->d_hdr + first;
    a.steps = c->d_steps + (uint64_t)first * c->step_cap;
    a.offs = c->d_offs + (uint64_t)first * c->step_cap;
    a.cumulative = c->d_cum;
    a.total = c->d_total;
    a.cumulative64 = c->d_cum64;
    a.reserved = c->g.reserved_rings_per_band;
    a.ref_reserved = c->g.reserved_rings_per_band;
    a.half_bands = c->g.computable_points_count;
    return a;
}

// Orders, on the GPU, every sequence of constant-table launches on one device:
// each sequence waits for the previous one (whatever stream it ran on) and
// becomes the one the next sequence waits for.
struct DeviceConstLock {
    static std::mutex &mutex() {
        static std::mutex m;
        return m;
    }
    static cudaEvent_t &last(int device) {
        static cudaEvent_t events[64] = {};
        return events[device & 63];
    }
    std::lock_guard<std::mutex> guard;
    cudaStream_t stream;
    int device;
    cudaError_t error = cudaSuccess;
    DeviceConstLock(int dev, cudaStream_t s) : guard(mutex()), stream(s), device(dev) {
        cudaEvent_t &ev = last(device);
        if (!ev) error = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (error == cudaSuccess) error = cudaStreamWaitEvent(stream, ev, 0);
    }
    ~DeviceConstLock() {
        if (error == cudaSuccess) cudaEventRecord(last(device), stream);
    }
};

// Sweep implementation for surface-only runs: the persistent work-queue
// kernel (default), per-sector constant-table launches, or the one-launch
// shared-memory kernel.  TVS_SWEEP_IMPL=queue|const|smem selects one for
// comparisons; ring output always uses the shared-memory kernel.
enum class SweepImpl { Queue, Const, Smem };

SweepImpl sweep_impl() {
    static SweepImpl v = [] {
        const char *e = getenv("TVS_SWEEP_IMPL");
        if (e && !strcmp(e, "const")) return SweepImpl::Const;
        if (e && !strcmp(e, "smem")) return SweepImpl::Smem;
        return SweepImpl::Queue;
    }();
    return v;
}

// Device ring buffer of `slots` u32 per band (the reference's reservation for
// its layout, compact_slots for the compact stream), the spill list and the
// counters; grown when a later call needs more slots.
int ensure_rings(tvs_context *c, uint32_t slots) {
    if (slots == 0)
        return fail(c, TVS_ERR_RING_OVERFLOW,
                    "no ring slots are reserved (rings_per_km * line of sight < 1 slot): the "
                    "reference's first ring write is out of bounds (kernel.rs:307)");
    const uint64_t need = c->g.total_bands * (uint64_t)slots;
    cudaError_t e = cudaSuccess;
    if (need > c->ring_capacity) {
        if (c->d_rings) {
            cudaFree(c->d_rings);
            c->device_bytes -= c->ring_capacity * sizeof(uint32_t);
            c->d_rings = nullptr;
            c->ring_capacity = 0;
        }
        e = cudaMalloc(&c->d_rings, std::max<uint64_t>(need, 1) * sizeof(uint32_t));
        if (e == cudaSuccess) {
            c->ring_capacity = std::max<uint64_t>(need, 1);
            c->device_bytes += c->ring_capacity * sizeof(uint32_t);
        }
    }
    if (e == cudaSuccess && !c->d_spill) {
        c->spill_cap = kSpillCap;
        e = cudaMalloc(&c->d_spill, (size_t)c->spill_cap * sizeof(uint4));
        if (e == cudaSuccess) e = cudaMalloc(&c->d_counters, 4 * sizeof(uint32_t));
        if (e == cudaSuccess) c->device_bytes += (size_t)c->spill_cap * sizeof(uint4) + 4 * sizeof(uint32_t);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, e == cudaErrorMemoryAllocation ? TVS_ERR_OUT_OF_MEMORY : TVS_ERR_CUDA,
                    std::string("ring buffer allocation: ") + cudaGetErrorString(e));
    }
    return TVS_OK;
}

int ensure_plain_scratch(tvs_context *c) {
    if (c->d_sf) return TVS_OK;
    const uint64_t n = (uint64_t)(c->row_end - c->row_begin) * c->g.tvs_width;
    TVS_CUDA(c, cudaMalloc(&c->d_sf, std::max<uint64_t>(n, 1) * sizeof(float)));
    TVS_CUDA(c, cudaMalloc(&c->d_sb, std::max<uint64_t>(n, 1) * sizeof(float)));
    c->device_bytes += 2 * std::max<uint64_t>(n, 1) * sizeof(float);
    return TVS_OK;
}

int enqueue_shape(tvs_context *c, uint32_t first, uint32_t count) {
    tvs::ShapeArgs a = shape_args(c, first);
    TVS_CUDA(c, tvs::launch_shape(a, count, c->stream));
    c->launches++;
    bool any = false;
    for (uint32_t s = first; s < first + count && s < tvs::kSectorSteps; s++) any |= c->installed[s];
    if (any) {  // installed tables replace the computed shapes of their sectors
        const uint64_t bds = c->g.band_deltas_size;
        TVS_CUDA(c, tvs::launch_shape_tables(a, count, c->d_tab_deltas + first * bds,
                                             c->d_tab_dists + first * bds, c->d_installed + first,
                                             c->stream));
        c->launches++;
    }
    for (uint32_t s = first; s < first + count && s < tvs::kSectorSteps; s++) c->pending[s] = true;
    return TVS_OK;
}

// This context as the one-DEM descriptor of the queue sweep, tiled for the
// context's configuration (uploaded again only when the configuration changes).
tvs::QueueDem queue_dem(const tvs_context *c) {
    tvs::QueueDem d{};
    d.elev = c->d_elev;
    d.quad = c->d_quad;
    d.quad_copy = tvs::quad_copy_elems(c->g.width, c->g.height);
    d.width = c->g.width;
    d.tvs_width = c->g.tvs_width;
    d.los = c->g.max_los_as_points;
    d.row_begin = c->row_begin;
    d.row_end = c->row_end;
    d.observer_height = c->p.observer_height;
    d.step_cap = c->step_cap;
    d.hdr = c->d_hdr;
    d.steps = c->d_steps;
    d.offs = c->d_offs;
    d.dtab = c->d_dtab;
    d.cumulative = c->d_cum;
    d.total = c->d_total;
    d.cumulative64 = c->d_cum64;
    d.hmax = c->d_hmax;
    d.bmax = c->d_bmax;
    d.bmax_w = c->bmax_w;
    d.bmax_h = c->bmax_h;
    return d;
}

// The split layout a launch runs: the quad layout needs the context's
// row-interleaved copies, else its tiling runs from the plain DEM.
int runnable_layout(const tvs_context *c, int layout) {
    return layout == tvs::kQuadLayout && !c->d_quad ? tvs::kQuadFallback : layout;
}

int upload_queue_dem(tvs_context *c) {
    const tvs::QueueConfig &q = c->qcfg, &u = c->qcfg_uploaded;
    if (q.px == u.px && q.py == u.py && q.layout == u.layout) return TVS_OK;
    tvs::QueueDem d = queue_dem(c);
    uint32_t done_total = 0;
    tvs::queue_tile(&d, 1, q, &c->q_tiles_per_sector, &done_total);
    TVS_CUDA(c, cudaMemcpyAsync(c->d_qdem, &d, sizeof d, cudaMemcpyHostToDevice, c->stream));
    c->qcfg_uploaded = q;
    return TVS_OK;
}

// The queue descriptor of this context tiled for the ring sweep's split
// layout: the context's own when its configuration is a split layout, else
// one for the precision's default split layout.
int ring_queue_dem(tvs_context *c, const tvs::QueueDem **dem, uint32_t *tiles, int *layout) {
    if (c->qcfg.layout != 0) {
        int rc = upload_queue_dem(c);
        if (rc) return rc;
        *dem = c->d_qdem;
        *tiles = c->q_tiles_per_sector;
        *layout = c->qcfg.layout;
        return TVS_OK;
    }
    const tvs::QueueConfig q = tvs::default_split_config((int)c->p.precision);
    if (!c->d_qdem_rings) {
        TVS_CUDA(c, cudaMalloc(&c->d_qdem_rings, sizeof(tvs::QueueDem)));
        c->device_bytes += sizeof(tvs::QueueDem);
        tvs::QueueDem d = queue_dem(c);
        uint32_t done_total = 0;
        tvs::queue_tile(&d, 1, q, &c->q_ring_tiles, &done_total);
        TVS_CUDA(c, cudaMemcpy(c->d_qdem_rings, &d, sizeof d, cudaMemcpyHostToDevice));
        c->ring_layout = (uint32_t)q.layout;
    }
    *dem = c->d_qdem_rings;
    *tiles = c->q_ring_tiles;
    *layout = (int)c->ring_layout;
    return TVS_OK;
}

// Sweep sectors [first, first+count) (slots == angles).  ring_slots != 0:
// count is 1 and the sector's ring records go to d_rings with ring_slots u32
// per band (the reference's reservation for its layout, compact_slots for the
// compact stream).
int enqueue_sweep(tvs_context *c, uint32_t first, uint32_t count, uint32_t ring_slots) {
    const bool rings = ring_slots != 0;
    if (c->p.sweep_kernel == TVS_SWEEP_PLAIN) {
        int rc = ensure_plain_scratch(c);
        if (rc) return rc;
        for (uint32_t s = first; s < first + count; s++) {
            tvs::PlainArgs a{};
            a.elev = c->d_elev;
            a.width = c->g.width;
            a.tvs_width = c->g.tvs_width;
            a.los = c->g.max_los_as_points;
            a.row_begin = c->row_begin;
            a.row_end = c->row_end;
            a.observer_height = c->p.observer_height;
            a.band_deltas_size = c->g.band_deltas_size;
            a.hdr = c->d_hdr + s;
            a.deltas = c->d_deltas + (uint64_t)s * c->g.band_deltas_size;
            a.dists = c->d_dists + (uint64_t)s * c->g.band_deltas_size;
            a.sf = c->d_sf;
            a.sb = c->d_sb;
            a.reserved = rings ? ring_slots : c->g.reserved_rings_per_band;
            a.half_bands = c->g.computable_points_count;
            if (rings) {
                a.rings = c->d_rings;
                a.spill = c->d_spill;
                a.spill_cap = c->spill_cap;
                a.counters = c->d_counters;
            }
            TVS_CUDA(c, tvs::launch_sweep_plain(a, c->stream));
            const uint64_t off = (uint64_t)c->row_begin * c->g.tvs_width;
            const uint64_t n = (uint64_t)(c->row_end - c->row_begin) * c->g.tvs_width;
            TVS_CUDA(c, tvs::launch_combine(c->d_cum + off, c->d_total + off, c->d_sf, c->d_sb,
                                            n, c->stream));
            c->launches += 2;
        }
        return TVS_OK;
    }
    const uint32_t n_steps =
        c->g.band_steps_filled + std::min(c->g.band_deltas_size - c->g.band_steps_filled, 2u);
    const SweepImpl impl = sweep_impl();
    if (rings && c->p.precision != TVS_PRECISION_FP64 && impl == SweepImpl::Queue) {
        // ring records from the direction-split sweep itself
        const tvs::QueueDem *dem = nullptr;
        uint32_t tiles = 0;
        int layout = 0;
        int rc = ring_queue_dem(c, &dem, &tiles, &layout);
        if (rc) return rc;
        tvs::QueueArgs q{};
        q.dems = dem;
        q.n_dems = 1;
        q.first_sector = first;
        q.n_sectors = count;
        q.tiles_per_sector = tiles;
        q.max_step_cap = c->step_cap;
        q.queue = c->d_queue;
        q.done = c->d_done;
        q.done_total = tiles;
        q.done_cap = c->done_cap;
        q.error = c->d_error;
        q.spin_limit = c->spin_limit;
        q.held_tile = c->held_tile;
        q.rechecks = c->d_rechecks;
        q.diag = c->diag_on ? c->d_diag : nullptr;
        q.rings = c->d_rings;
        q.ring_reserved = ring_slots;
        q.ref_reserved = c->g.reserved_rings_per_band;
        q.half_bands = c->g.computable_points_count;
        q.spill = c->d_spill;
        q.spill_cap = c->spill_cap;
        q.ring_counters = c->d_counters;
        TVS_CUDA(c, tvs::launch_sweep_split(q, (int)c->p.precision, runnable_layout(c, layout),
                                            c->stream));
        c->launches++;
        return TVS_OK;
    }
    if (!rings && impl == SweepImpl::Queue) {
        int rc = upload_queue_dem(c);
        if (rc) return rc;
        tvs::QueueArgs q{};
        q.dems = c->d_qdem;
        q.n_dems = 1;
        q.first_sector = first;
        q.n_sectors = count;
        q.tiles_per_sector = c->q_tiles_per_sector;
        q.max_step_cap = c->step_cap;
        q.queue = c->d_queue;
        q.done = c->d_done;
        q.done_total = c->q_tiles_per_sector;
        q.done_cap = c->done_cap;
        q.error = c->d_error;
        q.spin_limit = c->spin_limit;
        q.held_tile = c->held_tile;
        q.rechecks = c->d_rechecks;
        q.diag = c->diag_on ? c->d_diag : nullptr;
        tvs::QueueConfig cfg = c->qcfg;
        cfg.layout = runnable_layout(c, cfg.layout);
        TVS_CUDA(c, tvs::launch_sweep_queue(q, (int)c->p.precision, cfg, c->stream));
        c->launches++;
        return TVS_OK;
    }
    if (!rings && impl == SweepImpl::Const && c->p.precision == TVS_PRECISION_EXACT32 &&
        n_steps <= tvs::kConstSteps) {
        // Per-sector launches read the step table from the module's constant
        // memory, which every context on the device shares: serialise those
        // launch sequences on the GPU timeline across contexts.
        DeviceConstLock lock(c->p.device, c->stream);
        if (lock.error != cudaSuccess) return cuda_fail(c, lock.error, "constant-table lock");
        for (uint32_t s = first; s < first + count; s++) {
            tvs::SweepArgs a = sweep_args(c, s, 1);
            TVS_CUDA(c, tvs::launch_sweep_const(a, (int)c->p.precision, n_steps, c->stream));
            c->launches++;
        }
        return TVS_OK;
    }
    if (c->p.precision == TVS_PRECISION_FP32)
        return fail(c, TVS_ERR_INVALID_ARGUMENT, "the FP32 form runs on the persistent sweep only");
    tvs::SweepArgs a = sweep_args(c, first, count);
    if (rings) {
        a.reserved = ring_slots;
        a.rings = c->d_rings;
        a.spill = c->d_spill;
        a.spill_cap = c->spill_cap;
        a.counters = c->d_counters;
    }
    TVS_CUDA(c, tvs::launch_sweep_engine(a, (int)c->p.precision, c->stream));
    c->launches++;
    return TVS_OK;
}

int header_status(tvs_context *c, uint32_t first, uint32_t count) {
    std::vector<tvs::ShapeHeader> h(count);
    TVS_CUDA(c, cudaMemcpyAsync(h.data(), c->d_hdr + first, count * sizeof(tvs::ShapeHeader),
                                cudaMemcpyDeviceToHost, c->stream));
    TVS_CUDA(c, cudaStreamSynchronize(c->stream));
    for (uint32_t i = 0; i < count; i++) {
        if (h[i].status == TVS_OK) continue;
        char b[256];
        const char *what = h[i].status == TVS_ERR_PATH_OUT_OF_DEM
                               ? "a band of sight walks off the DEM (kernel.rs:164 index out of "
                                 "bounds)"
                           : h[i].status == TVS_ERR_CAPACITY
                               ? "too many sector-order key ties for the shape stage"
                               : "shape stage failed";
        std::snprintf(b, sizeof b, "sector %u: %s", first + i, what);
        return fail(c, h[i].status, b);
    }
    return TVS_OK;
}

// The shape slots of sectors [first, first+count) for the per-sector calls:
// computed (one launch per run of missing sectors, one status check) once,
// then reused until a table is installed for the sector.
int ensure_shapes(tvs_context *c, uint32_t first, uint32_t count) {
    bool launched = false;
    for (uint32_t s = first; s < first + count;) {
        if (c->shape_ok[s]) {
            s++;
            continue;
        }
        uint32_t e = s;
        while (e < first + count && !c->shape_ok[e]) e++;
        int rc = enqueue_shape(c, s, e - s);
        if (rc) return rc;
        launched = true;
        s = e;
    }
    if (!launched) return TVS_OK;
    int rc = header_status(c, first, count);
    if (rc) return rc;
    for (uint32_t s = first; s < first + count; s++) c->shape_ok[s] = true;
    return TVS_OK;
}
int ensure_shape(tvs_context *c, uint32_t angle) { return ensure_shapes(c, angle, 1); }

// Copy one sector's ring records to the host and apply the spilled ids with
// the reference's sequential semantics: band k writes slots k*R .. k*R+n_k
// (kernel.rs:141-243), so an id past its own record lands in a later band's
// record unless that band's own (later) writes cover the slot.
int collect_rings(tvs_context *c, uint32_t *rings, uint64_t rings_len, tvs_sector_stats *st) {
    uint32_t cnt[4];
    TVS_CUDA(c, cudaMemcpyAsync(cnt, c->d_counters, sizeof cnt, cudaMemcpyDeviceToHost,
                                c->stream));
    TVS_CUDA(c, cudaMemcpyAsync(rings, c->d_rings, c->g.ring_slots_per_sector * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, c->stream));
    TVS_CUDA(c, cudaStreamSynchronize(c->stream));
    if (st) {
        st->overflow_bands = cnt[1];
        st->max_ring_ids = cnt[2];
        st->spill_entries = cnt[0];
    }
    if (cnt[0] == 0) return TVS_OK;
    if (cnt[0] > c->spill_cap)
        return fail(c, TVS_ERR_CAPACITY, "ring spill list capacity exceeded");
    std::vector<uint4> sp(cnt[0]);
    TVS_CUDA(c, cudaMemcpy(sp.data(), c->d_spill, cnt[0] * sizeof(uint4), cudaMemcpyDeviceToHost));
    std::sort(sp.begin(), sp.end(), [](const uint4 &x, const uint4 &y) {
        uint64_t kx = x.x | ((uint64_t)x.y << 32), ky = y.x | ((uint64_t)y.y << 32);
        return kx != ky ? kx < ky : x.z < y.z;
    });
    const uint64_t R = c->g.reserved_rings_per_band;
    const uint64_t limit = std::min<uint64_t>(rings_len, c->g.ring_slots_per_sector);
    for (const uint4 &s : sp) {
        const uint64_t kid = s.x | ((uint64_t)s.y << 32);
        const uint64_t at = kid * R + s.z;
        if (at >= limit) {
            char b[200];
            std::snprintf(b, sizeof b,
                          "ring records overflow the sector buffer (band %llu slot %u; "
                          "kernel.rs:307 index out of bounds): raise --rings-per-km",
                          (unsigned long long)kid, s.z);
            return fail(c, TVS_ERR_RING_OVERFLOW, b);
        }
        const uint64_t owner = at / R, q = at % R;
        if (q > rings[owner * R]) rings[at] = s.w;  // owner's own writes cover 0..n_owner
    }
    return TVS_OK;
}

}  // namespace

// Sets the text tvs_last_error(NULL) returns (used by entry points that have
// no context).
void tvs_set_create_error(const std::string &msg) { g_create_error = msg; }

namespace tvs_host {
tvs::ShapeArgs shape_args_of(tvs_context *c, uint32_t first_slot) { return shape_args(c, first_slot); }
tvs::QueueDem queue_dem_of(const tvs_context *c) { return queue_dem(c); }
int header_status_of(tvs_context *c, uint32_t first, uint32_t count) {
    return header_status(c, first, count);
}
int fail_of(tvs_context *c, int code, const std::string &msg) { return fail(c, code, msg); }
int enqueue_shape_of(tvs_context *c, uint32_t first, uint32_t count) {
    return enqueue_shape(c, first, count);
}
void drop_tvs_graph_of(tvs_context *c) { drop_tvs_graph(c); }
}  // namespace tvs_host

extern "C" {

int tvs_abi_version(void) { return TVS_ABI_VERSION; }

const char *tvs_last_error(const tvs_context *ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int tvs_compute_geometry(const tvs_params *params, tvs_geometry *out) {
    if (!params || !out) return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "null argument");
    std::string msg;
    int rc = derive_geometry(params, out, &msg);
    if (rc) return fail(nullptr, rc, msg);
    return TVS_OK;
}

int tvs_create(const tvs_params *params, const float *elevations, uint64_t n_elevations,
               tvs_context **out) {
    if (!params || !out) return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    tvs_geometry g;
    std::string msg;
    int rc = derive_geometry(params, &g, &msg);
    if (rc) return fail(nullptr, rc, msg);
    if (!elevations || n_elevations != g.size)
        return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "elevations must hold width*height values");
    if (params->precision > TVS_PRECISION_FP32 || params->sweep_kernel > TVS_SWEEP_PLAIN ||
        (params->sweep_kernel == TVS_SWEEP_PLAIN && params->precision != TVS_PRECISION_EXACT32))
        return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "unsupported precision/sweep-kernel pair");
    uint32_t rb = params->tvs_row_begin, re = params->tvs_row_end;
    if (rb == 0 && re == 0) re = g.tvs_height;
    if (rb > re || re > g.tvs_height)
        return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "tvs row range outside the computable grid");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, TVS_ERR_NO_DEVICE, "no CUDA device");
    }
    if (params->device < 0 || params->device >= ndev)
        return fail(nullptr, TVS_ERR_NO_DEVICE, "device ordinal out of range");

    // the MIXED64 sweep keeps the step of each chain's maximum in 16 bits
    if (params->precision == TVS_PRECISION_MIXED64 && params->sweep_kernel == TVS_SWEEP_ENGINE &&
        g.band_steps_filled + 2 > 0xffffu)
        return fail(nullptr, TVS_ERR_INVALID_ARGUMENT,
                    "MIXED64 supports band tables of up to 65535 steps");
    tvs_context *c = new tvs_context();
    c->p = *params;
    c->g = g;
    c->row_begin = rb;
    c->row_end = re;
    const uint64_t los = g.max_los_as_points;
    if (g.computable_points_count) {
        c->pov_min = (int64_t)(los * g.width + los);
        c->pov_max = (int64_t)((g.tvs_height - 1 + los) * g.width + (g.tvs_width - 1 + los));
    }
    c->step_cap = (g.band_steps_filled + 2 + 3) & ~3u;
    c->done_cap = tvs::queue_tiles_bound(g.tvs_width, re - rb);
    c->bmax_w = (g.width + tvs::kBlockMax - 1) / tvs::kBlockMax;
    c->bmax_h = (g.height + tvs::kBlockMax - 1) / tvs::kBlockMax;
    c->qcfg = tvs::default_queue_config((int)c->p.precision);
    auto bail = [&](cudaError_t e, const char *what) {
        std::string m = std::string(what) + ": " + cudaGetErrorString(e);
        int code = e == cudaErrorMemoryAllocation ? TVS_ERR_OUT_OF_MEMORY : TVS_ERR_CUDA;
        cudaGetLastError();
        free_all(c);
        delete c;
        return fail(nullptr, code, m);
    };
    cudaError_t e = cudaSetDevice(params->device);
    if (e != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate");
    const uint64_t count = std::max<uint64_t>(g.computable_points_count, 1);
    const uint32_t slots = tvs::kSectorSteps + 1;
    const uint64_t bds = std::max<uint32_t>(g.band_deltas_size, 1);
    struct { void **p; size_t bytes; } allocs[] = {
        {(void **)&c->d_elev, (g.size + tvs::kElevationPad) * sizeof(float)},
        {(void **)&c->d_cum, count * sizeof(float)},
        {(void **)&c->d_total, count * sizeof(float)},
        {(void **)&c->d_trig, slots * sizeof(tvs::SectorTrig)},
        {(void **)&c->d_hdr, slots * sizeof(tvs::ShapeHeader)},
        {(void **)&c->d_steps, (size_t)slots * c->step_cap * sizeof(float4)},
        {(void **)&c->d_offs, (size_t)slots * c->step_cap * sizeof(int2)},
        {(void **)&c->d_dtab, (size_t)slots * c->step_cap * sizeof(double4)},
        {(void **)&c->d_queue, sizeof(uint32_t)},
        {(void **)&c->d_done, (size_t)std::max<uint32_t>(c->done_cap, 1) * sizeof(uint32_t)},
        {(void **)&c->d_error, sizeof(int32_t)},
        {(void **)&c->d_hmax, sizeof(float)},
        {(void **)&c->d_bmax, (size_t)std::max<uint64_t>((uint64_t)c->bmax_w * c->bmax_h, 1) * sizeof(float)},
        {(void **)&c->d_rechecks, sizeof(unsigned long long)},
        {(void **)&c->d_diag, 4 * sizeof(unsigned long long)},
        {(void **)&c->d_qdem, sizeof(tvs::QueueDem)},
        {(void **)&c->d_deltas, (size_t)slots * bds * sizeof(int32_t)},
        {(void **)&c->d_dists, (size_t)slots * bds * sizeof(float)},
    };
    for (auto &a : allocs) {
        if ((e = cudaMalloc(a.p, a.bytes)) != cudaSuccess) return bail(e, "cudaMalloc");
        c->device_bytes += a.bytes;
    }
    if (params->precision == TVS_PRECISION_MIXED64 || params->precision == TVS_PRECISION_FP64) {
        if ((e = cudaMalloc(&c->d_cum64, count * sizeof(double))) != cudaSuccess)
            return bail(e, "cudaMalloc");
        c->device_bytes += count * sizeof(double);
    }
    // the quad layout's copies (4x the DEM); without them (FP64, the plain
    // kernel, a DEM past the 32-bit offsets, or no memory for them) the quad
    // layout's tiling runs from the plain DEM
    if (params->precision != TVS_PRECISION_FP64 && params->sweep_kernel == TVS_SWEEP_ENGINE &&
        tvs::quad_fits(g.width, g.height)) {
        const size_t qb = 4 * tvs::quad_copy_elems(g.width, g.height) * sizeof(float4);
        if (cudaMalloc(&c->d_quad, qb) == cudaSuccess) {
            c->device_bytes += qb;
        } else {
            cudaGetLastError();
            c->d_quad = nullptr;
        }
    }
    // Per-sector trigonometry on the host (glibc, as Rust std on linux-gnu):
    // axes.rs:95 shifts the angle in f32, axes.rs:127 adds 90 in f32.
    std::vector<tvs::SectorTrig> trig(slots);
    for (uint32_t s = 0; s < tvs::kSectorSteps; s++) {
        const float sight = (float)s + tvs::kSectorShift;
        const float sector = sight + 90.0f;
        trig[s].sight_sin = std::sin((double)sight * kRadsPerDeg);
        trig[s].sight_cos = std::cos((double)sight * kRadsPerDeg);
        trig[s].sector_sin = std::sin((double)sector * kRadsPerDeg);
        trig[s].sector_cos = std::cos((double)sector * kRadsPerDeg);
    }
    trig[tvs::kSectorSteps] = trig[0];
    if ((e = cudaMemcpy(c->d_trig, trig.data(), slots * sizeof(tvs::SectorTrig),
                        cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e, "cudaMemcpy trig");
    if ((e = cudaMemcpy(c->d_elev, elevations, g.size * sizeof(float), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return bail(e, "cudaMemcpy elevations");
    if ((e = cudaMemset(c->d_elev + g.size, 0, tvs::kElevationPad * sizeof(float))) != cudaSuccess)
        return bail(e, "cudaMemset elevation padding");
    if ((e = tvs::launch_max_abs(c->d_elev, g.size, params->observer_height, c->d_hmax, 0)) !=
            cudaSuccess ||
        (e = tvs::launch_block_max(c->d_elev, g.width, g.height, c->d_bmax, 0)) != cudaSuccess ||
        (c->d_quad && (e = tvs::launch_quad_copies(c->d_elev, g.width, g.height, c->d_quad, 0)) !=
                          cudaSuccess) ||
        (e = cudaDeviceSynchronize()) != cudaSuccess)
        return bail(e, "elevation range");
    if ((e = cudaMemset(c->d_hdr, 0, slots * sizeof(tvs::ShapeHeader))) != cudaSuccess ||
        (e = cudaMemset(c->d_error, 0, sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMemset(c->d_rechecks, 0, sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMemset(c->d_diag, 0, 4 * sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMemset(c->d_cum, 0, count * sizeof(float))) != cudaSuccess ||
        (e = cudaMemset(c->d_total, 0, count * sizeof(float))) != cudaSuccess)
        return bail(e, "cudaMemset");
    if (c->d_cum64 && (e = cudaMemset(c->d_cum64, 0, count * sizeof(double))) != cudaSuccess)
        return bail(e, "cudaMemset");
    *out = c;
    return TVS_OK;
}

void tvs_destroy(tvs_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->p.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    delete ctx;
}

int tvs_get_geometry(const tvs_context *ctx, tvs_geometry *out) {
    if (!ctx || !out) return TVS_ERR_INVALID_ARGUMENT;
    *out = ctx->g;
    return TVS_OK;
}

int tvs_set_elevations(tvs_context *ctx, const float *elevations, uint64_t n) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (!elevations || n != ctx->g.size)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "elevations must hold width*height values");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    TVS_CUDA(ctx, cudaMemcpyAsync(ctx->d_elev, elevations, n * sizeof(float),
                                  cudaMemcpyHostToDevice, ctx->stream));
    // the estimate windows of the MIXED64 and filtered exact-f32 sweeps
    TVS_CUDA(ctx, tvs::launch_max_abs(ctx->d_elev, n, ctx->p.observer_height, ctx->d_hmax,
                                      ctx->stream));
    TVS_CUDA(ctx, tvs::launch_block_max(ctx->d_elev, ctx->g.width, ctx->g.height, ctx->d_bmax,
                                        ctx->stream));
    if (ctx->d_quad)
        TVS_CUDA(ctx, tvs::launch_quad_copies(ctx->d_elev, ctx->g.width, ctx->g.height,
                                              ctx->d_quad, ctx->stream));
    return TVS_OK;
}

int tvs_axes(tvs_context *ctx, uint32_t angle, uint64_t first_rank, uint64_t count,
             uint32_t *sector_ordered, float *sight_distances) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    const uint64_t win = (uint64_t)std::min(ctx->g.width, ctx->g.height) *
                         std::min(ctx->g.width, ctx->g.height);
    if (angle >= tvs::kSectorSteps || first_rank + count > win)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "angle or rank range out of bounds");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    if (sector_ordered && count) {
        if (count > tvs::kCandidateCap)
            return fail(ctx, TVS_ERR_CAPACITY, "tvs_axes rank range exceeds the candidate capacity");
        uint32_t *d_ids = nullptr;
        TVS_CUDA(ctx, cudaMalloc(&d_ids, count * sizeof(uint32_t)));
        const uint32_t slot = tvs::kSectorSteps;  // scratch slot
        tvs::SectorTrig t;
        TVS_CUDA(ctx, cudaMemcpyAsync(&t, ctx->d_trig + angle, sizeof t, cudaMemcpyDeviceToHost,
                                      ctx->stream));
        TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        TVS_CUDA(ctx, cudaMemcpyAsync(ctx->d_trig + slot, &t, sizeof t, cudaMemcpyHostToDevice,
                                      ctx->stream));
        tvs::ShapeArgs a = shape_args(ctx, slot);
        a.sector_ids_out = d_ids;
        a.dbg_first = first_rank;
        a.dbg_count = count;
        cudaError_t e = tvs::launch_shape(a, 1, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sector_ordered, d_ids, count * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        cudaFree(d_ids);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "tvs_axes");
        int rc = header_status(ctx, slot, 1);
        if (rc) return rc;
    }
    if (sight_distances) {
        tvs::SectorTrig t;
        TVS_CUDA(ctx, cudaMemcpy(&t, ctx->d_trig + angle, sizeof t, cudaMemcpyDeviceToHost));
        // The same device projection the shape stage uses (axes.rs:154-189).
        float *d_out = nullptr;
        TVS_CUDA(ctx, cudaMalloc(&d_out, ctx->g.size * sizeof(float)));
        cudaError_t e = tvs::launch_sight_distances(t, ctx->g.width, ctx->g.height, d_out,
                                                    ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sight_distances, d_out, ctx->g.size * sizeof(float),
                                cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        cudaFree(d_out);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "tvs_axes sight distances");
    }
    return TVS_OK;
}

int tvs_band_shape(tvs_context *ctx, uint32_t angle, int32_t *band_deltas, float *band_distances,
                   uint32_t *band_steps_filled) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (angle >= tvs::kSectorSteps) return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "angle >= 180");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    int rc = enqueue_shape(ctx, angle, 1);
    if (rc) return rc;
    const uint64_t bds = ctx->g.band_deltas_size;
    if (band_deltas && bds)
        TVS_CUDA(ctx, cudaMemcpyAsync(band_deltas, ctx->d_deltas + angle * bds,
                                      bds * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (band_distances && bds)
        TVS_CUDA(ctx, cudaMemcpyAsync(band_distances, ctx->d_dists + angle * bds,
                                      bds * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    tvs::ShapeHeader h;
    TVS_CUDA(ctx, cudaMemcpyAsync(&h, ctx->d_hdr + angle, sizeof h, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (band_steps_filled) *band_steps_filled = h.n_filled;
    if (h.status == TVS_ERR_CAPACITY || h.status == TVS_ERR_SHAPE) return header_status(ctx, angle, 1);
    return TVS_OK;
}

int tvs_compute_sector(tvs_context *ctx, uint32_t angle, float *cumulative_surfaces,
                       uint32_t *rings, uint64_t rings_len, tvs_sector_stats *stats) {
    if (!ctx || !cumulative_surfaces) return TVS_ERR_INVALID_ARGUMENT;
    if (angle >= tvs::kSectorSteps) return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "angle >= 180");
    if (rings && rings_len < ctx->g.ring_slots_per_sector)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "rings_len is smaller than one sector's slots");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    const uint64_t count = ctx->g.computable_points_count;
    if (count)
        TVS_CUDA(ctx, cudaMemcpyAsync(ctx->d_cum, cumulative_surfaces, count * sizeof(float),
                                      cudaMemcpyHostToDevice, ctx->stream));
    // FP64/MIXED64 accumulate in double within the sector, from the caller's f32
    if (ctx->d_cum64 && count)
        TVS_CUDA(ctx, tvs::launch_widen(ctx->d_cum, ctx->d_cum64, count, ctx->stream));
    const uint32_t R = ctx->g.reserved_rings_per_band;
    if (rings) {
        int rc = ensure_rings(ctx, R);
        if (rc) return rc;
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_rings, 0,
                                      ctx->g.ring_slots_per_sector * sizeof(uint32_t), ctx->stream));
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), ctx->stream));
    }
    int rc = ensure_shape(ctx, angle);
    if (rc) return rc;
    rc = enqueue_sweep(ctx, angle, 1, rings ? R : 0);
    if (rc) return rc;
    if (count)
        TVS_CUDA(ctx, cudaMemcpyAsync(cumulative_surfaces, ctx->d_cum, count * sizeof(float),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->angle = angle;
        stats->band_steps_filled = ctx->g.band_steps_filled;
    }
    if (rings) {
        rc = collect_rings(ctx, rings, rings_len, stats);
        if (rc) return rc;
    }
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TVS_OK;
}

int tvs_compute_sectors_rings(tvs_context *ctx, uint32_t first_angle, uint32_t n_sectors,
                              float *cumulative_surfaces, uint64_t *total_ids,
                              tvs_sector_stats *stats) {
    if (!ctx || !cumulative_surfaces || !total_ids) return TVS_ERR_INVALID_ARGUMENT;
    if (n_sectors == 0 || first_angle >= tvs::kSectorSteps ||
        n_sectors > tvs::kSectorSteps - first_angle)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "sectors outside 0..179 (or none)");
    // several sectors in one launch: the direction-split sweep only
    if (n_sectors > 1 && (ctx->p.precision == TVS_PRECISION_FP64 ||
                          ctx->p.sweep_kernel == TVS_SWEEP_PLAIN || sweep_impl() != SweepImpl::Queue))
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT,
                    "ring records of several sectors per call need the persistent split sweep "
                    "(not FP64 or the plain kernel)");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    ctx->rc_valid = false;
    const uint64_t count = ctx->g.computable_points_count;
    const uint64_t recs = ctx->g.total_bands * n_sectors;  // records of this call
    const uint64_t nb = tvs::ring_scan_blocks(recs);
    if (!ctx->d_rc_offsets || recs > ctx->rc_records_cap) {
        if (ctx->d_rc_offsets) {
            cudaFree(ctx->d_rc_offsets);
            cudaFree(ctx->d_rc_blocks);
            ctx->device_bytes -= (ctx->rc_records_cap + 1 + tvs::ring_scan_blocks(ctx->rc_records_cap) + 1) *
                                 sizeof(uint64_t);
            ctx->d_rc_offsets = nullptr;
            ctx->d_rc_blocks = nullptr;
            ctx->rc_records_cap = 0;
        }
        TVS_CUDA(ctx, cudaMalloc(&ctx->d_rc_offsets, (recs + 1) * sizeof(uint64_t)));
        TVS_CUDA(ctx, cudaMalloc(&ctx->d_rc_blocks, (nb + 1) * sizeof(uint64_t)));
        ctx->rc_records_cap = recs;
        ctx->device_bytes += (recs + 1 + nb + 1) * sizeof(uint64_t);
    }
    {
        int rc = ensure_shapes(ctx, first_angle, n_sectors);
        if (rc) return rc;
    }
    // The sweep writes up to `slots` ids per band in place and the rest to the
    // spill list.  When the sectors spill more than the list holds, the slots
    // per band double and the call runs again from the caller's surfaces (a
    // band has at most n_steps + 2 ids, so this ends).
    const uint32_t most = ctx->g.band_steps_filled + 4;
    uint32_t R = 0, cnt[4];
    uint64_t total = 0;
    int rc = TVS_OK;
    for (;;) {
        R = std::min(ctx->compact_slots, most);
        rc = ensure_rings(ctx, R * n_sectors);  // [sector][band][R]
        if (rc) return rc;
        if (count)
            TVS_CUDA(ctx, cudaMemcpyAsync(ctx->d_cum, cumulative_surfaces, count * sizeof(float),
                                          cudaMemcpyHostToDevice, ctx->stream));
        if (ctx->d_cum64 && count)
            TVS_CUDA(ctx, tvs::launch_widen(ctx->d_cum, ctx->d_cum64, count, ctx->stream));
        // Every band the split sweep covers writes its count (slot 0) and its
        // ids; the slots past a band's count are never read.  A row shard
        // leaves the other bands unwritten (their counts must read 0), and the
        // other sweeps write only where they have ids.
        if (ctx->row_begin != 0 || ctx->row_end != ctx->g.tvs_height ||
            ctx->p.sweep_kernel == TVS_SWEEP_PLAIN || ctx->p.precision == TVS_PRECISION_FP64 ||
            sweep_impl() != SweepImpl::Queue)
            TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_rings, 0, recs * R * sizeof(uint32_t), ctx->stream));
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), ctx->stream));
        rc = enqueue_sweep(ctx, first_angle, n_sectors, R);
        if (rc) return rc;
        // the record lengths (slot 0 holds a band's whole count, spilled ids
        // included) are scanned before the spill check: one wait for both
        TVS_CUDA(ctx, tvs::launch_ring_count(ctx->d_rings, recs, R, ctx->d_rc_blocks, ctx->stream));
        TVS_CUDA(ctx, cudaMemcpyAsync(cnt, ctx->d_counters, sizeof cnt, cudaMemcpyDeviceToHost,
                                      ctx->stream));
        TVS_CUDA(ctx, cudaMemcpyAsync(&total, ctx->d_rc_blocks + nb, sizeof total,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (cnt[0] <= ctx->spill_cap) break;
        if (R >= most)
            return fail(ctx, TVS_ERR_CAPACITY, "ring spill list capacity exceeded");
        ctx->compact_slots = std::min(2 * ctx->compact_slots, most);
    }
    if (count)
        TVS_CUDA(ctx, cudaMemcpyAsync(cumulative_surfaces, ctx->d_cum, count * sizeof(float),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->angle = first_angle;
        stats->band_steps_filled = ctx->g.band_steps_filled;
        stats->overflow_bands = cnt[1];
        stats->max_ring_ids = cnt[2];
        stats->spill_entries = cnt[0];
    }
    if (total > ctx->rc_ids_cap) {
        if (ctx->d_rc_ids) {
            cudaFree(ctx->d_rc_ids);
            ctx->device_bytes -= ctx->rc_ids_cap * sizeof(uint32_t);
            ctx->d_rc_ids = nullptr;
            ctx->rc_ids_cap = 0;
        }
        // twice the need: sectors' record counts vary, and a reallocation
        // (free + malloc of gigabytes) costs more than the spare memory
        const uint64_t cap = 2 * total;
        TVS_CUDA(ctx, cudaMalloc(&ctx->d_rc_ids, std::max<uint64_t>(cap, 1) * sizeof(uint32_t)));
        ctx->rc_ids_cap = std::max<uint64_t>(cap, 1);
        ctx->device_bytes += ctx->rc_ids_cap * sizeof(uint32_t);
    }
    if (recs == 0)
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_rc_offsets, 0, sizeof(uint64_t), ctx->stream));
    TVS_CUDA(ctx, tvs::launch_ring_gather(ctx->d_rings, recs, R, ctx->d_rc_blocks, ctx->d_spill,
                                          cnt[0], ctx->d_rc_offsets, ctx->d_rc_ids, ctx->stream));
    ctx->launches += 2;
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->rc_total = total;
    ctx->rc_records = recs;
    ctx->rc_valid = true;
    *total_ids = total;
    return TVS_OK;
}

int tvs_compute_sector_rings(tvs_context *ctx, uint32_t angle, float *cumulative_surfaces,
                             uint64_t *total_ids, tvs_sector_stats *stats) {
    if (ctx && angle >= tvs::kSectorSteps) return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "angle >= 180");
    return tvs_compute_sectors_rings(ctx, angle, 1, cumulative_surfaces, total_ids, stats);
}

int tvs_read_ring_records(tvs_context *ctx, uint64_t *band_offsets, uint32_t *ids) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (!ctx->rc_valid)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "no ring records: call tvs_compute_sector_rings");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    if (band_offsets)
        TVS_CUDA(ctx, cudaMemcpyAsync(band_offsets, ctx->d_rc_offsets,
                                      (ctx->rc_records + 1) * sizeof(uint64_t),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    if (ids && ctx->rc_total)
        TVS_CUDA(ctx, cudaMemcpyAsync(ids, ctx->d_rc_ids, ctx->rc_total * sizeof(uint32_t),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TVS_OK;
}

int tvs_device_reset(tvs_context *ctx) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    const uint64_t count = std::max<uint64_t>(ctx->g.computable_points_count, 1);
    TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_cum, 0, count * sizeof(float), ctx->stream));
    TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_total, 0, count * sizeof(float), ctx->stream));
    if (ctx->d_cum64)
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_cum64, 0, count * sizeof(double), ctx->stream));
    return TVS_OK;
}

int tvs_device_shape_sectors(tvs_context *ctx, uint32_t first_angle, uint32_t count) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (first_angle + count > tvs::kSectorSteps)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "sector range beyond 180");
    if (count == 0) return TVS_OK;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    return enqueue_shape(ctx, first_angle, count);
}

int tvs_device_sweep_sectors(tvs_context *ctx, uint32_t first_angle, uint32_t count) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (first_angle + count > tvs::kSectorSteps)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "sector range beyond 180");
    if (count == 0) return TVS_OK;
    for (uint32_t s = first_angle; s < first_angle + count; s++)
        if (!ctx->pending[s])
            return fail(ctx, TVS_ERR_INVALID_ARGUMENT,
                        "sweep of a sector whose shape stage has not run");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    return enqueue_sweep(ctx, first_angle, count, 0);
}

int tvs_device_run_sectors(tvs_context *ctx, uint32_t first_angle, uint32_t count) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    ctx->launches = 0;
    int rc = tvs_device_shape_sectors(ctx, first_angle, count);
    if (rc) return rc;
    return tvs_device_sweep_sectors(ctx, first_angle, count);
}

int tvs_device_finish(tvs_context *ctx) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int rc = TVS_OK;
    for (uint32_t s = 0; s < tvs::kSectorSteps && rc == TVS_OK; s++) {
        if (!ctx->pending[s]) continue;
        uint32_t e = s;
        while (e < tvs::kSectorSteps && ctx->pending[e]) e++;
        rc = header_status(ctx, s, e - s);
        s = e - 1;
    }
    for (bool &p : ctx->pending) p = false;
    int32_t err = 0;
    TVS_CUDA(ctx, cudaMemcpy(&err, ctx->d_error, sizeof err, cudaMemcpyDeviceToHost));
    if (err != 0) {
        TVS_CUDA(ctx, cudaMemset(ctx->d_error, 0, sizeof err));
        if (rc == TVS_OK)
            rc = fail(ctx, err, "sweep work queue: a tile's dependency wait gave up "
                                "(iteration limit); results of this run are incomplete");
    }
    return rc;
}

int tvs_read_surfaces(tvs_context *ctx, float *cumulative_out, float *total_out) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    const uint64_t count = ctx->g.computable_points_count;
    if (cumulative_out && count)
        TVS_CUDA(ctx, cudaMemcpyAsync(cumulative_out, ctx->d_cum, count * sizeof(float),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    if (total_out && count)
        TVS_CUDA(ctx, cudaMemcpyAsync(total_out, ctx->d_total, count * sizeof(float),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TVS_OK;
}

const float *tvs_device_cumulative(const tvs_context *ctx) { return ctx ? ctx->d_cum : nullptr; }

int tvs_set_sweep_config(tvs_context *ctx, const tvs_sweep_config *cfg) {
    if (!ctx || !cfg) return TVS_ERR_INVALID_ARGUMENT;
    tvs::QueueConfig c{cfg->points_x, cfg->points_y, cfg->packed != 0, cfg->prefetch != 0, cfg->layout};
    if (!tvs::queue_config_valid(c))
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "unsupported points-per-thread shape");
    if (c.layout != 0 && ctx->p.precision == TVS_PRECISION_FP64)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "sweep layouts 1-9 are not available for FP64");
    if (c.layout == 0 && ctx->p.precision == TVS_PRECISION_FP32)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "the FP32 form runs on sweep layouts 1-9 only");
    if (c.px != ctx->qcfg.px || c.py != ctx->qcfg.py || c.packed != ctx->qcfg.packed ||
        c.prefetch != ctx->qcfg.prefetch || c.layout != ctx->qcfg.layout)
        drop_tvs_graph(ctx);
    ctx->qcfg = c;
    return TVS_OK;
}

int tvs_get_sweep_config(const tvs_context *ctx, tvs_sweep_config *cfg) {
    if (!ctx || !cfg) return TVS_ERR_INVALID_ARGUMENT;
    cfg->points_x = ctx->qcfg.px;
    cfg->points_y = ctx->qcfg.py;
    cfg->packed = ctx->qcfg.packed;
    cfg->prefetch = ctx->qcfg.prefetch;
    cfg->layout = ctx->qcfg.layout;
    return TVS_OK;
}

int tvs_autotune(tvs_context *ctx, uint32_t sample_sectors, tvs_sweep_config *chosen) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    if (sample_sectors == 0 || sample_sectors > tvs::kSectorSteps)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "sample_sectors must be in [1, 180]");
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    const bool exact = ctx->p.precision == TVS_PRECISION_EXACT32;
    const bool f64 = ctx->p.precision == TVS_PRECISION_FP64;
    const bool fp32 = ctx->p.precision == TVS_PRECISION_FP32;
    const tvs::QueueConfig cands[] = {{1, 1, 0, 0, 0}, {2, 1, 0, 0, 0}, {4, 1, 0, 0, 0},
                                      {2, 2, 0, 0, 0}, {2, 1, 1, 0, 0}, {4, 1, 1, 0, 0},
                                      {1, 1, 0, 1, 0}, {2, 1, 0, 1, 0}, {4, 1, 0, 1, 0},
                                      {2, 2, 0, 1, 0}, {4, 1, 0, 0, 1}, {4, 1, 0, 0, 2},
                                      {4, 1, 0, 0, 3}, {4, 1, 0, 0, 4}, {4, 1, 0, 0, 5},
                                      {4, 1, 0, 0, 6}, {4, 1, 0, 0, 7}, {4, 1, 0, 0, 8},
                                      {4, 1, 0, 0, 9}};
    cudaEvent_t t0, t1;
    TVS_CUDA(ctx, cudaEventCreate(&t0));
    TVS_CUDA(ctx, cudaEventCreate(&t1));
    float best = 1e30f;
    tvs::QueueConfig best_cfg = ctx->qcfg;
    int rc = enqueue_shape(ctx, 0, sample_sectors);
    for (const tvs::QueueConfig &c : cands) {
        if (rc) break;
        if ((c.packed && !exact) || (c.layout != 0 && f64) || (c.layout == 0 && fp32)) continue;
        ctx->qcfg = c;
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && rc == TVS_OK; rep++) {  // the first run warms up
            cudaEventRecord(t0, ctx->stream);
            rc = enqueue_sweep(ctx, 0, sample_sectors, 0);
            cudaEventRecord(t1, ctx->stream);
            if (rc == TVS_OK && cudaEventSynchronize(t1) != cudaSuccess)
                rc = fail(ctx, TVS_ERR_CUDA, "autotune run failed");
            if (rc == TVS_OK) cudaEventElapsedTime(&ms, t0, t1);
        }
        if (rc == TVS_OK && ms < best) {
            best = ms;
            best_cfg = c;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    ctx->qcfg = best_cfg;
    drop_tvs_graph(ctx);
    for (bool &p : ctx->pending) p = false;
    if (rc) return rc;
    if (chosen) tvs_get_sweep_config(ctx, chosen);
    return TVS_OK;
}

int tvs_set_queue_wait(tvs_context *ctx, uint32_t spin_limit, uint32_t held_tile) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    ctx->spin_limit = spin_limit ? spin_limit : tvs::kDefaultSpinLimit;
    ctx->held_tile = held_tile;
    drop_tvs_graph(ctx);
    return TVS_OK;
}

int tvs_set_sweep_counters(tvs_context *ctx, int enable) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    if (enable)
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_diag, 0, 4 * sizeof(unsigned long long), ctx->stream));
    if ((enable != 0) != ctx->diag_on) drop_tvs_graph(ctx);
    ctx->diag_on = enable != 0;
    return TVS_OK;
}

int tvs_read_sweep_counters(tvs_context *ctx, uint64_t *counters) {
    if (!ctx || !counters) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    unsigned long long v[4];
    TVS_CUDA(ctx, cudaMemcpyAsync(v, ctx->d_diag, sizeof v, cudaMemcpyDeviceToHost, ctx->stream));
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < 4; i++) counters[i] = v[i];
    return TVS_OK;
}

int tvs_device_run_tvs(tvs_context *ctx) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    // reset, the 180 shape stages and the sweep, with the stage events
    // (captured, the events become event-record nodes of the graph)
    auto enqueue_tvs = [&](bool captured) -> int {
        auto record = [&](cudaEvent_t ev) {
            return captured ? cudaEventRecordWithFlags(ev, ctx->stream, cudaEventRecordExternal)
                            : cudaEventRecord(ev, ctx->stream);
        };
        TVS_CUDA(ctx, record(ctx->ev_begin));
        int rc = tvs_device_reset(ctx);
        if (rc == TVS_OK) rc = enqueue_shape(ctx, 0, tvs::kSectorSteps);
        if (rc) return rc;
        TVS_CUDA(ctx, record(ctx->ev_shaped));
        rc = enqueue_sweep(ctx, 0, tvs::kSectorSteps, 0);
        if (rc) return rc;
        TVS_CUDA(ctx, record(ctx->ev_swept));
        return TVS_OK;
    };
    if (!ctx->tvs_exec) {
        // The first call runs the sequence with plain launches (which loads the
        // kernels and sets their launch attributes outside any capture), then
        // captures the same sequence for the later calls.
        for (cudaEvent_t *ev : {&ctx->ev_begin, &ctx->ev_shaped, &ctx->ev_swept})
            if (!*ev) TVS_CUDA(ctx, cudaEventCreate(ev));
        if (ctx->p.sweep_kernel == TVS_SWEEP_PLAIN) {
            int rc = ensure_plain_scratch(ctx);
            if (rc) return rc;
        }
        ctx->launches = 0;
        int rc = enqueue_tvs(false);
        for (uint32_t s = 0; s < tvs::kSectorSteps; s++) ctx->pending[s] = true;
        if (rc) return rc;
        const uint64_t plain = ctx->launches;
        TVS_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_tvs(true);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc != TVS_OK) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->tvs_exec, g, 0);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            ctx->tvs_exec = nullptr;
            cudaGetLastError();
            return cuda_fail(ctx, e, "capturing the total-viewshed graph");
        }
        ctx->tvs_graph = g;
        ctx->tvs_graph_launches = ctx->launches - plain;
        ctx->launches = plain;
        return TVS_OK;
    }
    TVS_CUDA(ctx, cudaGraphLaunch(ctx->tvs_exec, ctx->stream));
    for (uint32_t s = 0; s < tvs::kSectorSteps; s++) ctx->pending[s] = true;
    ctx->launches = ctx->tvs_graph_launches;
    return TVS_OK;
}

int tvs_last_run_times(tvs_context *ctx, float *shape_ms, float *sweep_ms) {
    if (!ctx || !ctx->ev_begin) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    TVS_CUDA(ctx, cudaEventSynchronize(ctx->ev_swept));
    float a = 0.0f, b = 0.0f;
    TVS_CUDA(ctx, cudaEventElapsedTime(&a, ctx->ev_begin, ctx->ev_shaped));
    TVS_CUDA(ctx, cudaEventElapsedTime(&b, ctx->ev_shaped, ctx->ev_swept));
    if (shape_ms) *shape_ms = a;
    if (sweep_ms) *sweep_ms = b;
    return TVS_OK;
}

int tvs_measure_l1_load(int32_t device, double *bytes_per_second) {
    if (!bytes_per_second) return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "null argument");
    cudaError_t e = cudaSetDevice(device);
    double v = 0.0;
    if (e == cudaSuccess) e = tvs::measure_l1_load(&v);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, TVS_ERR_CUDA, std::string("l1 load: ") + cudaGetErrorString(e));
    }
    *bytes_per_second = v;
    return TVS_OK;
}

int tvs_read_rechecks(tvs_context *ctx, uint64_t *count, int reset) {
    if (!ctx || !count) return TVS_ERR_INVALID_ARGUMENT;
    TVS_CUDA(ctx, cudaSetDevice(ctx->p.device));
    unsigned long long v = 0;
    TVS_CUDA(ctx, cudaMemcpyAsync(&v, ctx->d_rechecks, sizeof v, cudaMemcpyDeviceToHost, ctx->stream));
    TVS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (reset) TVS_CUDA(ctx, cudaMemset(ctx->d_rechecks, 0, sizeof v));
    *count = v;
    return TVS_OK;
}

void *tvs_stream(const tvs_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

uint64_t tvs_last_launch_count(const tvs_context *ctx) { return ctx ? ctx->launches : 0; }

uint64_t tvs_device_bytes(const tvs_context *ctx) { return ctx ? ctx->device_bytes : 0; }

int tvs_run(tvs_context *ctx, float *cumulative_out, float *total_out, int want_rings,
            tvs_sector_callback callback, void *user) {
    if (!ctx) return TVS_ERR_INVALID_ARGUMENT;
    int rc = tvs_device_reset(ctx);
    if (rc) return rc;
    if (!want_rings) {
        rc = tvs_device_run_tvs(ctx);
        if (rc) return rc;
        rc = tvs_device_finish(ctx);
        if (rc) return rc;
        if (callback)
            for (uint32_t s = 0; s < tvs::kSectorSteps; s++) {
                tvs_sector_stats st{};
                st.angle = s;
                st.band_steps_filled = ctx->g.band_steps_filled;
                if (callback(user, s, nullptr, 0, &st)) break;
            }
        return tvs_read_surfaces(ctx, cumulative_out, total_out);
    }
    if ((ctx->p.precision == TVS_PRECISION_MIXED64 || ctx->p.precision == TVS_PRECISION_FP64) &&
        !ctx->d_cum64)
        return fail(ctx, TVS_ERR_INVALID_ARGUMENT, "FP64 context without FP64 accumulator");
    rc = ensure_rings(ctx, ctx->g.reserved_rings_per_band);
    if (rc) return rc;
    std::vector<uint32_t> host_rings(ctx->g.ring_slots_per_sector);
    for (uint32_t s = 0; s < tvs::kSectorSteps; s++) {
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_rings, 0,
                                      ctx->g.ring_slots_per_sector * sizeof(uint32_t), ctx->stream));
        TVS_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), ctx->stream));
        rc = enqueue_shape(ctx, s, 1);
        if (rc) return rc;
        rc = header_status(ctx, s, 1);
        if (rc) return rc;
        rc = enqueue_sweep(ctx, s, 1, ctx->g.reserved_rings_per_band);
        if (rc) return rc;
        tvs_sector_stats st{};
        st.angle = s;
        st.band_steps_filled = ctx->g.band_steps_filled;
        rc = collect_rings(ctx, host_rings.data(), host_rings.size(), &st);
        if (rc) return rc;
        if (callback && callback(user, s, host_rings.data(), host_rings.size(), &st)) break;
    }
    return tvs_read_surfaces(ctx, cumulative_out, total_out);
}

int tvs_selftest_division(int32_t device, uint64_t n, uint64_t seed, uint64_t *mismatches) {
    if (!mismatches) return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "null argument");
    cudaError_t e = cudaSetDevice(device);
    unsigned long long *d = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&d, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = tvs::launch_selftest_division(n, seed, d, 0);
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, TVS_ERR_CUDA, std::string("selftest: ") + cudaGetErrorString(e));
    }
    *mismatches = h;
    return TVS_OK;
}

int tvs_measure_fp32_issue(int32_t device, double *instructions_per_second) {
    if (!instructions_per_second) return fail(nullptr, TVS_ERR_INVALID_ARGUMENT, "null argument");
    cudaError_t e = cudaSetDevice(device);
    double v = 0.0;
    if (e == cudaSuccess) e = tvs::measure_fp32_issue(&v);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, TVS_ERR_CUDA, std::string("fp32 issue: ") + cudaGetErrorString(e));
    }
    *instructions_per_second = v;
    return TVS_OK;
}

}  // extern "C"
