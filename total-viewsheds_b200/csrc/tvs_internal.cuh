// tvs_internal.cuh -- shared definitions of the B200 total-viewshed engine.
//
// Data layout in HBM (one context):
//   elevations   f32 [height][width]            uploaded once (main.rs:51-56)
//   cumulative   f32 [tvs_height][tvs_width]     kernel.rs:254 running sum
//   total        f32 [tvs_height][tvs_width]     compute.rs:206-214 heatmap total
//   per sector s (180 slots):
//     ShapeHeader                                status + step counts + offset bounds
//     StepTable  float4 {1/d, d, d/R, d*tan1} [step_cap]   sweep constants per step
//     StepOff    int2   {offset, flags}        [step_cap]   forward DEM-id offset
//     deltas i32 / distances f32 [band_deltas_size]          band_of_sight.rs output
//   rings        u32 [total_bands * reserved]   reference ring layout (one sector)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tvs {

// kernel.rs:13,17,21 and axes.rs:47
constexpr float kMaxAngle = -2000.0f;
constexpr float kTanOneRad = 0.0174533f;
constexpr float kEarthRadiusSquared = 12742000.0f;
// Side of the DEM blocks whose maximum elevation bounds the direction-split
// sweep's segments (kBlockMax x kBlockMax points per block).
#ifndef TVS_BLOCK_MAX
#define TVS_BLOCK_MAX 16
#endif
constexpr uint32_t kBlockMax = TVS_BLOCK_MAX;

// Four row-interleaved copies of a DEM for the quad split layout: copy c
// holds rows c + 4g .. c + 4g + 3 of group g as one float4 per column, so the
// four points of view of a lane, in consecutive rows, read one aligned 16-byte
// vector at every step whatever the step's row offset.  Rows past the DEM are
// zero; the groups reach the rows that a tile past the grid's last row
// addresses (up to H + 30), and kQuadPad float4 after them the columns past a
// row's end.  The sweep's step offsets are 32-bit byte offsets, so the four
// copies must lie within 2^31 bytes (quad_fits).
constexpr int kQuadLayout = 9;     // the split layout that reads them
constexpr int kQuadFallback = 7;   // the same tiling from the plain DEM
constexpr uint32_t kQuadPad = 64;
__host__ __device__ constexpr uint32_t quad_groups(uint32_t height) { return (height + 48) / 4 + 2; }
__host__ __device__ constexpr uint64_t quad_copy_elems(uint32_t width, uint32_t height) {
    return ((uint64_t)quad_groups(height) * width + kQuadPad + 15) & ~(uint64_t)15;
}
__host__ __device__ constexpr bool quad_fits(uint32_t width, uint32_t height) {
    return 4 * quad_copy_elems(width, height) * 16 < (1ull << 31);
}

#ifdef __CUDACC__
// The FP64 sweep's per-step values from the step's f32 distance d
// (kernel.rs:175,216 in double): {1/d, d/R, d*tan1, d}.  The shape stage
// tabulates them; sweeps short of shared memory recompute them from d.
__device__ __forceinline__ double4 fp64_step(float d) {
    const double dd = (double)d;
    return make_double4(__drcp_rn(dd), __ddiv_rn(dd, 12742000.0), __dmul_rn(dd, 0.0174533), dd);
}
#endif
// Iterations (256 ns sleeps) a work-queue dependency wait may take before it
// gives up with TVS_ERR_TIMEOUT: about 2-4 s, against a real wait of one
// work item (about a millisecond).
constexpr uint32_t kDefaultSpinLimit = 1u << 23;
constexpr float kSectorShift = 0.001f;
constexpr uint32_t kSectorSteps = 180;

// Shape-stage capacities (shared memory of the one-CTA-per-sector kernel).
constexpr uint32_t kShapeThreads = 1024;
constexpr uint32_t kCandidateCap = 16384;  // sector-order candidates (u64 each)
constexpr uint32_t kWindowCap = 8192;      // band_samples (u64 each)

// Step flags.
constexpr int kStepSlowDivide = 1;  // distance outside the table-division domain

struct SectorTrig {
    double sight_sin, sight_cos;    // sin/cos(rad(angle + 0.001))         axes.rs:107
    double sector_sin, sector_cos;  // sin/cos(rad((angle + 0.001) + 90))  axes.rs:127
};

struct ShapeHeader {
    int32_t status;        // tvs_status of this sector's shape stage
    uint32_t n_filled;     // delta-table entries the reference fills
    uint32_t n_steps;      // steps the sweep evaluates (filled + <= 2 zero-distance)
    uint32_t n_candidates; // diagnostics: sector-order candidates gathered
    int64_t min_off;       // min over {0, offsets of evaluated steps}
    int64_t max_off;
    uint32_t n_fast;       // steps before the first kStepSlowDivide step
    uint32_t pad;
};

// Per-sector sweep launches read their step table from constant memory, so
// every table value is a warp-uniform operand (no shared-memory loads, no
// per-lane table addressing).  2560 steps cover band_steps_filled + 2 for a
// line of sight of up to ~4360 cells.
constexpr uint32_t kConstSteps = 2560;
// Zero floats after the elevations: a constant-table sweep thread covers up to
// 8 columns 32 apart, so lanes past the computable grid read at most
// 32*8 + 32 floats beyond the last point of view's band (discarded results).
constexpr uint32_t kElevationPad = 32 * 8 + 64;

struct ShapeArgs {
    uint32_t width, height;
    uint64_t size;
    // The square the shape is built on: the whole DEM when it is square, the
    // central min(W, H) square otherwise (columns [x0, x0+win), rows [y0, y0+win)).
    uint32_t win, x0, y0;
    uint32_t band_size, band_deltas_size, band_samples;
    uint32_t first_angle;      // sector of blockIdx.x == 0
    uint32_t step_cap;         // per-sector stride of the step tables
    // Extremes of the point-of-view ids (every computable point).
    int64_t pov_min, pov_max;
    const SectorTrig *trig;    // [sectors]
    ShapeHeader *hdr;          // [sectors]
    float4 *steps;             // [sectors][step_cap]
    int2 *offs;                // [sectors][step_cap]
    double4 *dtab;             // [sectors][step_cap] FP64 {1/d, d/R, d*tan1, d}
    int32_t *deltas;           // [sectors][band_deltas_size]
    float *dists;              // [sectors][band_deltas_size]
    // Optional debug outputs for sector 0 of the launch (tvs_axes):
    uint32_t *sector_ids_out;  // ranks [dbg_first, dbg_first + dbg_count)
    uint64_t dbg_first, dbg_count;
};

struct SweepArgs {
    const float *elev;
    uint32_t width;
    uint32_t tvs_width;
    uint32_t row_begin, row_end;   // computable rows of this context
    uint32_t los;                  // max_los_as_points
    float observer_height;
    uint32_t n_sectors;
    uint32_t step_cap;
    const ShapeHeader *hdr;        // [n_sectors]
    const float4 *steps;
    const int2 *offs;
    float *cumulative;             // f32 [tvs_h * tvs_w]
    float *total;                  // f32 heatmap total (nullable)
    double *cumulative64;          // MIXED64/FP64 accumulation (nullable)
    // Ring output (one sector per launch when non-null).
    uint32_t *rings;
    uint32_t reserved;             // slots per band in `rings`
    uint32_t ref_reserved;         // the reference's slots per band (overflow statistics)
    uint64_t half_bands;           // computable_points_count
    uint4 *spill;                  // {kernel id lo, kernel id hi, slot, value}
    uint32_t spill_cap;
    uint32_t *counters;            // [0] spill count [1] overflow bands [2] max ids
};

// Persistent sweep over a (sector, DEM, tile) work queue (sweep_queue.cu).
// One DEM of the queue: a context is a batch of one.
struct QueueDem {
    const float *elev;
    const float4 *quad;                // the row-interleaved copies (nullable)
    uint64_t quad_copy;                // float4 per copy
    uint32_t width, tvs_width, los;
    uint32_t row_begin, row_end;
    float observer_height;
    uint32_t step_cap;
    const ShapeHeader *hdr;            // per sector slot (absolute slot index)
    const float4 *steps;
    const int2 *offs;
    const double4 *dtab;               // FP64 tables {1/d, d/R, d*tan1, d} (double)
    float *cumulative;
    float *total;                      // nullable
    double *cumulative64;              // FP64/MIXED64 only
    const float *hmax;                 // MIXED64: max |elevation| + |observer height|
    const float *bmax;                 // max elevation of each kBlockMax^2 block of the DEM
    uint32_t bmax_w, bmax_h;           // blocks per row, block rows
    uint32_t tiles_x, tiles_y;         // set by queue_tile
    uint32_t tile_base;                // first item of this DEM within a sector
    uint32_t done_base;                // this DEM's per-tile counters in `done`
};

struct QueueArgs {
    const QueueDem *dems;              // device array, tile_base ascending
    uint32_t n_dems;
    uint32_t first_sector, n_sectors;  // absolute sector slots
    uint32_t tiles_per_sector;         // sum of tiles_x * tiles_y
    uint32_t max_step_cap;
    uint32_t *queue;                   // [1] next work item
    uint32_t *done;                    // [done_cap] sectors completed per tile
    uint32_t done_total, done_cap;
    int32_t *error;                    // TVS_ERR_TIMEOUT when a wait gives up
    uint32_t spin_limit;
    uint32_t held_tile;                // failure-detection test hook: this tile
                                       // counter (done_base + tile) never advances
                                       // (0xFFFFFFFF: none)
    unsigned long long *rechecks;      // re-decided comparisons (nullable)
    // Ring records of the direction-split sweeps (nullable; one sector per
    // launch): band k's count at rings[k * ring_reserved], its ids in slots
    // 1 .. ring_reserved - 1, further ids as {k lo, k hi, slot, id} in spill.
    uint32_t *rings;
    uint32_t ring_reserved;            // slots per band in `rings`
    uint32_t ref_reserved;             // the reference's slots per band (statistics)
    uint64_t half_bands;               // computable points of the whole grid
    uint4 *spill;
    uint32_t spill_cap;
    uint32_t *ring_counters;           // [0] spill entries [1] bands past ref_reserved
                                       // [2] most ids in one band
    // Diagnostics (nullable): [0] warp-steps swept, [1] warp-steps past the
    // first test, [2] warp-steps of the fast loop in all, [3] spare.
    unsigned long long *diag;
};

// Points of view per thread (columns px 32 apart, rows py 8 apart), the
// packed f32x2 arithmetic switch (exact f32 only), the elevation prefetch
// switch (the next step's loads issued before the current step computes) and
// the layout: 0 rows of 32 lanes sweeping both directions together, 1 the
// MIXED64 direction-split layout (8 x 4 lanes, px = 4 points 8 columns apart).
struct QueueConfig {
    int px, py, packed, prefetch, layout;
};

struct PlainArgs {
    const float *elev;
    uint32_t width, tvs_width, los;
    uint32_t row_begin, row_end;
    float observer_height;
    uint32_t band_deltas_size;
    const ShapeHeader *hdr;        // one sector
    const int32_t *deltas;
    const float *dists;
    float *sf, *sb;                // per-point band surfaces of the shard
    uint32_t *rings;
    uint32_t reserved;
    uint64_t half_bands;
    uint4 *spill;
    uint32_t spill_cap;
    uint32_t *counters;
};

// radsort's order-preserving f32 -> u32 key (total order, -0.0 < +0.0).
__host__ __device__ inline uint32_t f32_radix_key(float f) {
#ifdef __CUDA_ARCH__
    uint32_t bits = __float_as_uint(f);
#else
    uint32_t bits;
    __builtin_memcpy(&bits, &f, 4);
#endif
    uint32_t mask = (uint32_t)(-(int32_t)(bits >> 31)) | 0x80000000u;
    return bits ^ mask;
}

// Host launchers (shape.cu, sweep.cu).
// Compact ring records (rings_compact.cu): block sums of the record lengths
// (ring_scan_blocks(bands) + 1 entries, exclusive-scanned, total last), then
// the offsets and ids.
uint64_t ring_scan_blocks(uint64_t bands);
cudaError_t launch_ring_count(const uint32_t *rings, uint64_t bands, uint32_t reserved,
                              uint64_t *block_sums, cudaStream_t s);
cudaError_t launch_ring_gather(const uint32_t *rings, uint64_t bands, uint32_t reserved,
                               const uint64_t *block_sums, const uint4 *spill, uint32_t n_spill,
                               uint64_t *offsets, uint32_t *ids, cudaStream_t s);
// bmax[(y / kBlockMax) * bmax_w + x / kBlockMax] = max elevation of the block
// (NaN ignored; -inf for an all-NaN block).
cudaError_t launch_block_max(const float *elev, uint32_t width, uint32_t height, float *bmax,
                             cudaStream_t s);
// The quad layout's copies of a width x height DEM (4 * quad_copy_elems float4).
cudaError_t launch_quad_copies(const float *elev, uint32_t width, uint32_t height, float4 *quad,
                               cudaStream_t s);
cudaError_t launch_shape_tables(const ShapeArgs &a, uint32_t n_sectors, const int32_t *tab_deltas,
                                const float *tab_dists, const unsigned char *installed,
                                cudaStream_t s);
cudaError_t launch_shape(const ShapeArgs &a, uint32_t n_sectors, cudaStream_t s);
cudaError_t launch_sight_distances(const SectorTrig &t, uint32_t width, uint32_t height,
                                   float *out, cudaStream_t s);
cudaError_t launch_sweep_engine(const SweepArgs &a, int precision, cudaStream_t s);
// Raises kernel fn's dynamic shared-memory limit on the current device to at
// least smem bytes (never lowers it; thread-safe).
cudaError_t grow_smem_attribute(const void *fn, size_t smem);
// One sector per launch with the step table staged in constant memory
// (hdr/steps/offs point at that sector's tables; a.n_sectors must be 1).
cudaError_t launch_sweep_const(const SweepArgs &a, int precision, uint32_t n_steps,
                               cudaStream_t s);
cudaError_t launch_sweep_plain(const PlainArgs &a, cudaStream_t s);
cudaError_t launch_sweep_queue(const QueueArgs &a, int precision, const QueueConfig &c,
                               cudaStream_t s);
// The direction-split layouts 1-6 (sweep_split.cu): EXACT32, MIXED64 and
// FP32; ring records when a.rings is set (one sector).
cudaError_t launch_sweep_split(const QueueArgs &a, int precision, int layout, cudaStream_t s);
size_t split_smem_bytes(int precision, uint32_t step_cap);
uint32_t queue_tiles_bound(uint32_t tvs_width, uint32_t rows);
bool queue_config_valid(const QueueConfig &c);
QueueConfig default_queue_config(int precision);
// The precision's default direction-split layout (for the ring sweep when the
// context's own configuration is a row layout).
QueueConfig default_split_config(int precision);
// Sets tiles_x/tiles_y/tile_base/done_base of every DEM for the configuration.
void queue_tile(QueueDem *dems, uint32_t n_dems, const QueueConfig &c, uint32_t *tiles_per_sector,
                uint32_t *done_total);
cudaError_t launch_shape_batch(const ShapeArgs *d_args, uint32_t n_dems, uint32_t n_sectors,
                               cudaStream_t s);
cudaError_t launch_combine(float *cum, float *total, const float *sf, const float *sb,
                           uint64_t n, cudaStream_t s);
cudaError_t measure_fp32_issue(double *instructions_per_second);
cudaError_t measure_l1_load(double *bytes_per_second);
// y[i] = (double)x[i]
cudaError_t launch_widen(const float *x, double *y, uint64_t n, cudaStream_t s);
// out[0] = max |x[i]| + |add| over n floats (out must hold 1 float).
cudaError_t launch_max_abs(const float *x, uint64_t n, float add, float *out, cudaStream_t s);
cudaError_t launch_selftest_division(uint64_t n, uint64_t seed, unsigned long long *mismatches,
                                     cudaStream_t s);

}  // namespace tvs
