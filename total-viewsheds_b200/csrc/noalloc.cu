// noalloc.cu -- one sector of the total viewshed without allocating anything.
//
// Who needs this: callers that cannot call cudaMalloc at the moment they want
// a sector computed.
//  * Hosts whose device memory belongs to another allocator (a framework's
//    caching allocator, or a fixed memory pool that must account for every
//    byte on the device): a cudaMalloc behind its back would break its
//    accounting or fail once the pool has taken the memory.
//  * Real-time or embedded callers that forbid allocation after start-up,
//    because an allocation can block or fail at an arbitrary moment.
// tvs_compute_sector_noalloc takes device pointers for its inputs and outputs
// (elevations in, cumulative and total surfaces in/out) and keeps the sector's
// intermediate tables (trigonometry, shape header, step tables, deltas and
// distances) in the fixed array below.  It calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// The array is compiled into the library: every GPU that loads the library
// holds its 64 KiB until the process exits.  All calls on a device share it,
// and it keeps the last call's contents.  Calls that overlap on the GPU race
// on it; this entry point keeps its own calls from overlapping by holding a
// process-wide lock for the whole call and synchronising the stream before it
// returns.  The call runs on params->device: it makes that device current for
// the call and gives the caller back the device that was current before.  The
// first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "tvs.h"
#include "tvs_internal.cuh"

namespace {

// 64 KiB: the tables of a line of sight of up to ~1590 cells (the 3601^2
// precision configuration uses 1200).
constexpr size_t kScratchBytes = 64u << 10;

}  // namespace

// The scratch array.  In host code this name is a host-side stand-in for the
// symbol, not a device address: only the address cudaGetSymbolAddress returns
// for the current device may be handed to a kernel.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

void tvs_set_create_error(const std::string &msg);  // capi.cu: tvs_last_error(NULL)

namespace {

constexpr double kRadsPerDeg = 3.14159265358979323846 / 180.0;  // Rust f64::to_radians

std::mutex g_mutex;
void *g_scratch[256] = {};  // device address of the array, per device ordinal

int fail(int code, const std::string &msg) {
    tvs_set_create_error(msg);
    return code;
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Byte offsets of one sector's tables inside the scratch array.
struct ScratchLayout {
    size_t trig, hdr, steps, offs, dtab, deltas, dists, total;
    ScratchLayout(uint32_t cap, uint32_t bds) {
        trig = 0;
        hdr = trig + align256(sizeof(tvs::SectorTrig));
        steps = hdr + align256(sizeof(tvs::ShapeHeader));
        offs = steps + align256((size_t)cap * sizeof(float4));
        dtab = offs + align256((size_t)cap * sizeof(int2));
        deltas = dtab + align256((size_t)cap * sizeof(double4));
        dists = deltas + align256((size_t)bds * sizeof(int32_t));
        total = dists + align256((size_t)bds * sizeof(float));
    }
};

// Device address of the scratch array on the current device (looked up once
// per device, on the first call made with that device current).
int scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(TVS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 256) return fail(TVS_ERR_NO_DEVICE, "device ordinal out of range");
    if (!g_scratch[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(TVS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                          cudaGetErrorString(e));
        g_scratch[dev] = p;
    }
    *out = g_scratch[dev];
    return TVS_OK;
}

int run_sector(const tvs_params *params, const tvs_geometry &g, uint32_t rb, uint32_t re,
               uint32_t cap, const float *d_elevations, uint32_t angle, float *d_cumulative,
               float *d_total, cudaStream_t s);

}  // namespace

extern "C" int tvs_compute_sector_noalloc(const tvs_params *params, const float *d_elevations,
                                          uint32_t angle, float *d_cumulative, float *d_total,
                                          void *stream) {
    if (!params || !d_elevations || !d_cumulative)
        return fail(TVS_ERR_INVALID_ARGUMENT, "null argument");
    if (angle >= tvs::kSectorSteps) return fail(TVS_ERR_INVALID_ARGUMENT, "angle >= 180");
    if (params->precision != TVS_PRECISION_EXACT32)
        return fail(TVS_ERR_INVALID_ARGUMENT, "the no-allocation entry point computes exact f32 only");
    tvs_geometry g;
    int rc = tvs_compute_geometry(params, &g);  // DEM::new checks (sets the error text)
    if (rc) return rc;
    uint32_t rb = params->tvs_row_begin, re = params->tvs_row_end;
    if (rb == 0 && re == 0) re = g.tvs_height;
    if (rb > re || re > g.tvs_height)
        return fail(TVS_ERR_INVALID_ARGUMENT, "tvs row range outside the computable grid");

    // Layout of the scratch array for this geometry.
    const uint32_t cap = (g.band_steps_filled + 2 + 3) & ~3u;
    const ScratchLayout lay(cap, g.band_deltas_size);
    const size_t total = lay.total;
    if (total > kScratchBytes) {
        char b[256];
        std::snprintf(b, sizeof b,
                      "line of sight of %u cells needs %zu bytes of sector tables; the "
                      "no-allocation entry point has %zu (up to ~1590 cells): use tvs_create",
                      g.max_los_as_points, total, kScratchBytes);
        return fail(TVS_ERR_CAPACITY, b);
    }

    // Nothing to compute (a line of sight of exactly half the shorter side):
    // no device work, as a context would do for the same geometry.
    if (g.computable_points_count == 0 || rb == re) return TVS_OK;

    std::lock_guard<std::mutex> lock(g_mutex);
    // The call runs on params->device (the device of the caller's buffers and
    // stream) and gives the caller back the device that was current.
    int previous = 0;
    cudaError_t e = cudaGetDevice(&previous);
    if (e != cudaSuccess)
        return fail(TVS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (params->device != previous && (e = cudaSetDevice(params->device)) != cudaSuccess) {
        cudaGetLastError();
        return fail(TVS_ERR_NO_DEVICE, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    rc = run_sector(params, g, rb, re, cap, d_elevations, angle, d_cumulative, d_total,
                    static_cast<cudaStream_t>(stream));
    if (params->device != previous) cudaSetDevice(previous);
    return rc;
}

namespace {

int run_sector(const tvs_params *params, const tvs_geometry &g, uint32_t rb, uint32_t re,
               uint32_t cap, const float *d_elevations, uint32_t angle, float *d_cumulative,
               float *d_total, cudaStream_t s) {
    const uint32_t bds = g.band_deltas_size;
    const ScratchLayout lay(cap, bds);
    const size_t off_trig = lay.trig, off_hdr = lay.hdr, off_steps = lay.steps;
    const size_t off_offs = lay.offs, off_dtab = lay.dtab, off_deltas = lay.deltas;
    const size_t off_dists = lay.dists;
    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char *sc = static_cast<unsigned char *>(base);

    // axes.rs:95,127 angles (f32), glibc trigonometry as Rust std on linux-gnu.
    tvs::SectorTrig trig;
    const float sight = (float)angle + tvs::kSectorShift;
    const float sector = sight + 90.0f;
    trig.sight_sin = std::sin((double)sight * kRadsPerDeg);
    trig.sight_cos = std::cos((double)sight * kRadsPerDeg);
    trig.sector_sin = std::sin((double)sector * kRadsPerDeg);
    trig.sector_cos = std::cos((double)sector * kRadsPerDeg);

    tvs::ShapeArgs a{};
    a.width = g.width;
    a.height = g.height;
    a.size = g.size;
    a.win = std::min(g.width, g.height);
    a.x0 = (g.width - a.win) / 2;
    a.y0 = (g.height - a.win) / 2;
    a.band_size = g.band_size;
    a.band_deltas_size = bds;
    a.band_samples = g.band_samples;
    a.first_angle = angle;
    a.step_cap = cap;
    const uint64_t los = g.max_los_as_points;
    a.pov_min = (int64_t)(los * g.width + los);
    a.pov_max = (int64_t)((g.tvs_height - 1 + los) * g.width + (g.tvs_width - 1 + los));
    a.trig = reinterpret_cast<const tvs::SectorTrig *>(sc + off_trig);
    a.hdr = reinterpret_cast<tvs::ShapeHeader *>(sc + off_hdr);
    a.steps = reinterpret_cast<float4 *>(sc + off_steps);
    a.offs = reinterpret_cast<int2 *>(sc + off_offs);
    a.dtab = reinterpret_cast<double4 *>(sc + off_dtab);
    a.deltas = reinterpret_cast<int32_t *>(sc + off_deltas);
    a.dists = reinterpret_cast<float *>(sc + off_dists);

    // The shape stage overwrites every table the sweep reads; the header is
    // cleared first so a failed launch cannot leave the last call's status.
    cudaError_t e = cudaMemsetAsync(sc + off_hdr, 0, sizeof(tvs::ShapeHeader), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sc + off_trig, &trig, sizeof trig, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = tvs::launch_shape(a, 1, s);
    tvs::ShapeHeader h{};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&h, sc + off_hdr, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return fail(TVS_ERR_CUDA, std::string("no-allocation shape stage: ") + cudaGetErrorString(e));
    if (h.status != TVS_OK) {
        char b[160];
        std::snprintf(b, sizeof b, "sector %u: %s", angle,
                      h.status == TVS_ERR_PATH_OUT_OF_DEM
                          ? "a band of sight walks off the DEM (kernel.rs:164 index out of bounds)"
                          : "shape stage failed");
        return fail(h.status, b);
    }

    // The sweep reads only the tables above, the caller's elevations (active
    // lanes only) and the caller's surfaces.
    tvs::SweepArgs w{};
    w.elev = d_elevations;
    w.width = g.width;
    w.tvs_width = g.tvs_width;
    w.row_begin = rb;
    w.row_end = re;
    w.los = g.max_los_as_points;
    w.observer_height = params->observer_height;
    w.n_sectors = 1;
    w.step_cap = cap;
    w.hdr = a.hdr;
    w.steps = a.steps;
    w.offs = a.offs;
    w.cumulative = d_cumulative;
    w.total = d_total;
    w.reserved = g.reserved_rings_per_band;
    w.half_bands = g.computable_points_count;
    e = tvs::launch_sweep_engine(w, TVS_PRECISION_EXACT32, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return fail(TVS_ERR_CUDA, std::string("no-allocation sweep: ") + cudaGetErrorString(e));
    return TVS_OK;
}

}  // namespace
