/*
 * tvs.h -- C ABI of the B200 total-viewshed engine (libtvs_cuda.so).
 *
 * The reference (tombh/total-viewsheds) dispatches each sector to a backend in
 * Compute::compute_sector (crates/total-viewsheds/src/compute.rs:181-203); its
 * `ComputeType::Cuda` arm is `unimplemented!()` (compute.rs:197).  These entry
 * points are what that arm binds through a Rust `extern "C"` block (built by
 * build.rs): plain pointers and sizes, status codes, no exceptions or aborts
 * across the boundary.
 *
 * Ownership: the caller owns every pointer it passes; the library reads or
 * writes them before returning.  The library owns its device buffers.
 * Threading: one context per host thread; calls on one context are serialised
 * by the caller.  Each context owns one CUDA stream on its device.
 */
#ifndef TVS_H
#define TVS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TVS_ABI_VERSION 5

/* Status codes.  Negative values are errors; tvs_last_error() has the text. */
enum tvs_status {
    TVS_OK = 0,
    TVS_ERR_INVALID_ARGUMENT = -1,
    /* dem.rs:56-62: line of sight longer than half the DEM width. */
    TVS_ERR_LOS_TOO_LONG = -2,
    /* band_of_sight.rs:103-165: the shape window or strip falls outside the
     * sorted DEM (the reference panics on an index). */
    TVS_ERR_SHAPE = -3,
    /* kernel.rs:157-164: a band walks off the DEM (the reference panics on
     * elevations[dem_id]). */
    TVS_ERR_PATH_OUT_OF_DEM = -4,
    /* kernel.rs:302-309: ring records overflow past the end of the sector's
     * ring buffer (the reference panics on ring_data[index]). */
    TVS_ERR_RING_OVERFLOW = -5,
    TVS_ERR_CUDA = -6,
    TVS_ERR_NO_DEVICE = -7,
    TVS_ERR_OUT_OF_MEMORY = -8,
    /* An internal fixed-capacity buffer (shape candidates, ring spill list)
     * was too small for this input. */
    TVS_ERR_CAPACITY = -9,
    /* A device wait gave up after its iteration limit. */
    TVS_ERR_TIMEOUT = -10
};

/* Sweep arithmetic.  See kernel.rs:164-233 for the reference expression. */
enum tvs_precision {
    /* Bit-exact with the reference f32 kernel: surfaces and ring records. */
    TVS_PRECISION_EXACT32 = 0,
    /* FP32 fast path from reciprocal/curvature tables; every comparison within
     * 8 ulp of the running maximum is re-decided in FP64.  Visibility matches
     * the all-FP64 sweep; surfaces accumulate in FP64. */
    TVS_PRECISION_MIXED64 = 1,
    /* The all-FP64 sweep (angles, running maximum, surfaces in double). */
    TVS_PRECISION_FP64 = 2,
    /* The plain reciprocal-table FP32 form, the comparison baseline (no
     * counterpart in the reference): angle = fma(h - h_pov, RN(1/d), -RN(d/R))
     * in one rounding, f32 comparisons and surfaces.  Its visibility differs
     * from both the reference's f32 and from FP64 near ties. */
    TVS_PRECISION_FP32 = 3
};

/* Which sweep kernel runs. */
enum tvs_sweep_kernel {
    /* The tiled engine: one thread per point of view, both band directions
     * interleaved, step tables in shared memory. */
    TVS_SWEEP_ENGINE = 0,
    /* The plain port of the reference shader: one thread per band, IEEE
     * divisions, every step of the delta table.  The baseline (EXACT32 only). */
    TVS_SWEEP_PLAIN = 1
};

typedef struct tvs_params {
    uint32_t width;              /* DEM columns (Header.width, input.rs:98)          */
    uint32_t height;             /* DEM rows; the reference requires height == width */
    float scale;                 /* metres per cell (--scale, config.rs:51-53)       */
    uint32_t max_line_of_sight;  /* metres (--max-line-of-sight, config.rs:18-24)    */
    float rings_per_km;          /* --rings-per-km (config.rs:26-33)                  */
    float observer_height;       /* metres; compute.rs:41 hard-codes 1.8             */
    uint32_t precision;          /* enum tvs_precision                               */
    uint32_t sweep_kernel;       /* enum tvs_sweep_kernel                            */
    int32_t device;              /* CUDA device ordinal                              */
    uint32_t tvs_row_begin;      /* computable-grid rows handled by this context:    */
    uint32_t tvs_row_end;        /* [begin, end); 0,0 = every row                    */
} tvs_params;

/* Geometry derived as DEM::new (dem.rs:44-72) and Compute::new
 * (compute.rs:27-56, cfg(test) ring sizing) derive it. */
typedef struct tvs_geometry {
    uint32_t width;
    uint32_t height;
    uint32_t max_los_as_points;        /* dem.rs:53                               */
    uint32_t band_size;                /* dem.rs:78                               */
    uint32_t band_deltas_size;         /* band_of_sight.rs:54-58                  */
    uint32_t tvs_width;                /* dem.rs:82                               */
    uint32_t tvs_height;
    uint32_t reserved_rings_per_band;  /* compute.rs:94-98                        */
    uint32_t band_samples;             /* band_of_sight.rs:95                     */
    uint32_t band_steps_filled;        /* entries of the delta table the shape    */
                                       /* stage fills (band_of_sight.rs:158)      */
    uint64_t size;                     /* width * height                          */
    uint64_t computable_points_count;  /* dem.rs:87-115                           */
    uint64_t total_bands;              /* compute.rs:34                           */
    uint64_t ring_slots_per_sector;    /* total_bands * reserved_rings_per_band   */
} tvs_geometry;

typedef struct tvs_sector_stats {
    uint32_t angle;
    uint32_t band_steps_filled;
    uint32_t overflow_bands;     /* bands with more ring ids than reserved slots  */
    uint32_t max_ring_ids;       /* ring-record high-water mark (ids in one band) */
    uint64_t spill_entries;      /* ring ids written past their own record        */
} tvs_sector_stats;

typedef struct tvs_context tvs_context;

/* Called by tvs_run after each sector with that sector's ring records in the
 * reference layout (kernel.rs:141-145,243), or NULL when the callback asked
 * for none.  Return non-zero to stop the run. */
typedef int (*tvs_sector_callback)(void *user, uint32_t angle, const uint32_t *rings,
                                   uint64_t rings_len, const tvs_sector_stats *stats);

/* ---- lifetime -------------------------------------------------------- */

/* GPU::new (gpu.rs:55-61): validate the geometry, pick the device, allocate,
 * upload the elevations (row-major, width*height f32). */
int tvs_create(const tvs_params *params, const float *elevations, uint64_t n_elevations,
               tvs_context **out);
void tvs_destroy(tvs_context *ctx);
/* Last error text of ctx, or of the last failed tvs_create when ctx is NULL. */
const char *tvs_last_error(const tvs_context *ctx);
int tvs_abi_version(void);

/* DEM::new + Compute::new geometry, without a context or a GPU. */
int tvs_compute_geometry(const tvs_params *params, tvs_geometry *out);
int tvs_get_geometry(const tvs_context *ctx, tvs_geometry *out);

/* Replace the elevations (same size).  main.rs:51-56 converts i16 -> f32. */
int tvs_set_elevations(tvs_context *ctx, const float *elevations, uint64_t n_elevations);

/* ---- the per-sector stages ------------------------------------------- */

/* Axes::compute (axes.rs:103-130) restricted to what the shape needs:
 * sector_ordered[first_rank .. first_rank+count) (ids in sector order) and
 * the f32 sight distances of every point (nullable).  For a rectangular DEM
 * the order covers the central min(W, H) square the shape is built on. */
int tvs_axes(tvs_context *ctx, uint32_t angle, uint64_t first_rank, uint64_t count,
             uint32_t *sector_ordered, float *sight_distances);

/* DEM::compile_band_data (band_of_sight.rs:61-174): band_deltas_size entries;
 * entries past band_steps_filled are 0 as in the reference. */
int tvs_band_shape(tvs_context *ctx, uint32_t angle, int32_t *band_deltas,
                   float *band_distances, uint32_t *band_steps_filled);

/* A sector's band shape given as tables instead of computed, as when
 * Compute::load_or_compute_cache (compute.rs:118-162) loads it from the cache
 * (cache.rs:50-60).  Every later shape stage of that sector uses the first
 * band_deltas_size entries of band_deltas/band_distances (n entries given):
 * fewer than that -> TVS_ERR_SHAPE (the reference's kernel indexes past them);
 * tables that fill more steps than this width and line of sight ->
 * TVS_ERR_SHAPE.  tvs_band_shape then returns these tables.  Not used by
 * batches or tvs_compute_sector_noalloc. */
int tvs_set_band_shape(tvs_context *ctx, uint32_t angle, const int32_t *band_deltas,
                       const float *band_distances, uint64_t n);
/* Back to computed shapes for every sector. */
int tvs_clear_band_shapes(tvs_context *ctx);
/* The reference's shape cache (cache.rs:23-78) under state_directory (the
 * reference uses the OS state directory, main.rs:63):
 *   total-viewsheds/<width>/band_deltas/<angle>.bin   i32[band_deltas_size]
 *   total-viewsheds/<width>/distances/<angle>.bin     f32[band_deltas_size]
 * (raw, native-endian; a rectangular DEM uses <width>x<height>).  Load
 * installs every sector whose two files exist (tvs_set_band_shape rules) and
 * reports how many; save computes every sector's shape and writes its files,
 * skipping sectors whose two files exist unless overwrite != 0 (the reference
 * writes a sector's files when it had to compute them). */
int tvs_cache_load(tvs_context *ctx, const char *state_directory, uint32_t *sectors_loaded);
int tvs_cache_save(tvs_context *ctx, const char *state_directory, int overwrite);

/* Compute::compute_sector (compute.rs:181-203) for ComputeType::Cuda:
 * cumulative_surfaces [computable_points_count] is read, advanced by this
 * sector and written back (kernel.rs:254).  FP64 and MIXED64 contexts widen
 * the f32 input and accumulate the sector in double (tvs_run keeps double
 * across sectors).  rings (nullable) receives the
 * sector's ring records in the reference layout; rings_len must be at least
 * ring_slots_per_sector.  stats is nullable. */
int tvs_compute_sector(tvs_context *ctx, uint32_t angle, float *cumulative_surfaces,
                       uint32_t *rings, uint64_t rings_len, tvs_sector_stats *stats);

/* The sector's ring records as a compact stream instead of the reference's
 * reserved slots (kernel.rs:141-145,220-243,302-309, 2.08 GB per sector at
 * 3601^2 with mostly empty slots): band k's record (pov, closing, opening,
 * closing, ... -- the n ids after the reference's count slot, never truncated
 * by the reservation) is ids[band_offsets[k] .. band_offsets[k+1]).  This call
 * advances cumulative_surfaces as tvs_compute_sector does, keeps the records
 * on the device and returns their id count; tvs_read_ring_records copies
 * band_offsets [total_bands + 1] (u64) and ids [*total_ids] (either nullable).
 * No counterpart in the reference; the records equal its per-band records. */
int tvs_compute_sector_rings(tvs_context *ctx, uint32_t angle, float *cumulative_surfaces,
                             uint64_t *total_ids, tvs_sector_stats *stats);
/* Sectors [first_angle, first_angle + n_sectors) in one sweep launch, as
 * Compute::run's loop takes them (compute.rs:106-112): cumulative_surfaces
 * advances by every sector in order (FP64 and MIXED64 keep double between the
 * call's sectors, as tvs_run does), and the records of all of them form one
 * compact stream in which sector first_angle + s owns records
 * s * total_bands .. (s + 1) * total_bands - 1.  stats aggregates the sectors
 * (angle = first_angle).  More than one sector needs the persistent split
 * sweep (not FP64 or the plain kernel); the slots behind the stream take
 * n_sectors * total_bands * 64 u32 of device memory.  No counterpart in the
 * reference (it computes one sector per call). */
int tvs_compute_sectors_rings(tvs_context *ctx, uint32_t first_angle, uint32_t n_sectors,
                              float *cumulative_surfaces, uint64_t *total_ids,
                              tvs_sector_stats *stats);
/* The records of the last tvs_compute_sector_rings or tvs_compute_sectors_rings
 * call: band_offsets [records + 1] (records = n_sectors * total_bands) and
 * ids [*total_ids], either nullable. */
int tvs_read_ring_records(tvs_context *ctx, uint64_t *band_offsets, uint32_t *ids);

/* Compute::run (compute.rs:101-115): all 180 sectors.  cumulative_out and
 * total_out (the heatmap running total, compute.rs:206-214; nullable) have
 * computable_points_count entries.  callback (nullable) receives each
 * sector's ring records when want_rings != 0. */
int tvs_run(tvs_context *ctx, float *cumulative_out, float *total_out, int want_rings,
            tvs_sector_callback callback, void *user);

/* ---- device-resident form (inputs and outputs stay in HBM) ----------- */

/* Zero the device cumulative and running-total surfaces. */
int tvs_device_reset(tvs_context *ctx);
/* Enqueue sectors [first_angle, first_angle+count) on the context's stream
 * (no host synchronisation, no rings).  Errors surface at tvs_device_finish. */
int tvs_device_run_sectors(tvs_context *ctx, uint32_t first_angle, uint32_t count);
/* The two stages of tvs_device_run_sectors, for callers that time them apart:
 * the shape stage (one CTA per sector) and the sweep (one launch). */
int tvs_device_shape_sectors(tvs_context *ctx, uint32_t first_angle, uint32_t count);
int tvs_device_sweep_sectors(tvs_context *ctx, uint32_t first_angle, uint32_t count);
/* One whole total viewshed on the context's stream: zero the surfaces, the
 * shape stage of all 180 sectors and one persistent sweep over them.  The
 * first call runs these as plain launches and captures them in a CUDA graph;
 * later calls replay the graph (one launch).  A new sweep configuration,
 * installed shapes, wait settings or counters drop the graph.  No counterpart
 * in the reference (its Compute::run loops sectors on the host,
 * compute.rs:101-115). */
int tvs_device_run_tvs(tvs_context *ctx);
/* Device times of the last tvs_device_run_tvs: the reset and shape stage, and
 * the sweep (waits for it to finish). */
int tvs_last_run_times(tvs_context *ctx, float *shape_ms, float *sweep_ms);
/* Wait for the stream and report the first error of the sectors enqueued
 * since the last tvs_device_finish, if any. */
int tvs_device_finish(tvs_context *ctx);
/* Copy the device surfaces to the host (either pointer nullable). */
int tvs_read_surfaces(tvs_context *ctx, float *cumulative_out, float *total_out);
/* MIXED64: number of sample comparisons re-decided in FP64 since the last
 * reset (reset != 0 clears the counter after reading). */
int tvs_read_rechecks(tvs_context *ctx, uint64_t *count, int reset);
/* Device pointer of the float32 cumulative surfaces, for zero-copy callers. */
const float *tvs_device_cumulative(const tvs_context *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time on it. */
void *tvs_stream(const tvs_context *ctx);
/* Number of kernels the last tvs_device_run_sectors call enqueued. */
uint64_t tvs_last_launch_count(const tvs_context *ctx);
/* Bytes of device memory the context holds (its peak: buffers are only ever
 * added, the ring buffers on the first run that asks for ring records). */
uint64_t tvs_device_bytes(const tvs_context *ctx);

/* Failure detection of the persistent sweep (no counterpart in the reference,
 * which has no device waits).  A work item waits for its tile's previous
 * sector before adding its surfaces; the wait sleeps in steps of ~256 ns and
 * gives up after spin_limit steps (0 = the default, about 2 s): the item's
 * writes are skipped, later waits give up at once, and tvs_device_finish
 * returns TVS_ERR_TIMEOUT.  held_tile (0xFFFFFFFF = none) is a test hook:
 * that tile's completion counter never advances, so the wait of its next
 * sector cannot be satisfied.  Applies to this context's later sweeps. */
int tvs_set_queue_wait(tvs_context *ctx, uint32_t spin_limit, uint32_t held_tile);

/* Sweep counters of the direction-split layouts, for roofline accounting (no
 * counterpart in the reference).  enable != 0 zeroes them and counts the
 * later sweeps, 0 stops counting (the counts stay readable); read gives [0] warp-steps swept (not skipped by the segment
 * bounds), [1] warp-steps that passed the first test, [2] warp-steps of the
 * table-division loop in all (swept or skipped), [3] 0. */
int tvs_set_sweep_counters(tvs_context *ctx, int enable);
int tvs_read_sweep_counters(tvs_context *ctx, uint64_t *counters);

/* ---- sweep configuration and autotuning ------------------------------ */

/* Points of view per thread of the persistent sweep: points_x columns 32
 * apart times points_y rows 8 apart (1x1, 2x1, 4x1, 2x2, 8x1), i.e. a CTA tile
 * of 32*points_x x 8*points_y points; packed != 0 selects the packed f32x2
 * arithmetic (exact f32 only); prefetch != 0 issues the next step's elevation
 * loads before the current step's arithmetic (not with packed).  layout
 * L in 1..9 (MIXED64, EXACT32 and FP32, with points 4x1) sweeps one direction
 * at a time, evaluating angles exactly only where a warp's first test passes:
 * a warp holds LX = 8, 16, 32 (L = 1, 2, 3 and again 4, 5, 6; 32 and 16 for
 * L = 7, 8) columns x 32/LX rows of lanes; each lane has four points of view
 * LX columns apart (L <= 3, tiles of 4 LX x 256/LX points), 2 x 2 of them, LX
 * columns and 32/LX rows apart (L = 4..6, tiles of 2 LX x 512/LX), or four of
 * them in one column, 32/LX rows apart (L = 7, 8, tiles of LX x 1024/LX).
 * L = 9 is L = 7's tiling read from four row-interleaved copies of the DEM
 * (one 16-byte load per lane and step; the context holds the copies, 4x the
 * DEM, when the DEM fits 32-bit offsets into them, else L = 9 runs as L = 7).
 * Defaults: the fastest split layout per precision on one B200; rows 2x1 for
 * FP64 (the only layout it runs).  Results do not depend on any of them. */
typedef struct tvs_sweep_config {
    int32_t points_x;
    int32_t points_y;
    int32_t packed;
    int32_t prefetch;
    int32_t layout;
} tvs_sweep_config;

int tvs_set_sweep_config(tvs_context *ctx, const tvs_sweep_config *cfg);
int tvs_get_sweep_config(const tvs_context *ctx, tvs_sweep_config *cfg);
/* Times every candidate configuration on sectors [0, sample_sectors) of this
 * context and keeps the fastest (returned in *chosen, nullable).  The device
 * surfaces are undefined afterwards: reset before the next run. */
int tvs_autotune(tvs_context *ctx, uint32_t sample_sectors, tvs_sweep_config *chosen);

/* ---- batches of DEM tiles --------------------------------------------- */

/* No counterpart in the reference (which runs one DEM per process).  Many DEM
 * tiles of uneven, possibly rectangular size: every run computes all 180
 * sectors of every tile with one shape launch and one persistent sweep,
 * captured in a CUDA graph on the first run and replayed afterwards.
 * params[i] and elevations[i] describe tile i (same device and precision for
 * every tile). */
typedef struct tvs_batch tvs_batch;

int tvs_batch_create(const tvs_params *params, const float *const *elevations, uint32_t n_dems,
                     tvs_batch **out);
void tvs_batch_destroy(tvs_batch *batch);
const char *tvs_batch_last_error(const tvs_batch *batch);
uint32_t tvs_batch_size(const tvs_batch *batch);
int tvs_batch_geometry(const tvs_batch *batch, uint32_t dem, tvs_geometry *out);
int tvs_batch_set_sweep_config(tvs_batch *batch, const tvs_sweep_config *cfg);
int tvs_batch_get_sweep_config(const tvs_batch *batch, tvs_sweep_config *cfg);
/* As tvs_autotune, on the whole batch (drops the captured graph). */
int tvs_batch_autotune(tvs_batch *batch, uint32_t sample_sectors, tvs_sweep_config *chosen);
/* Enqueue one full run (graph replay) on the batch's stream. */
int tvs_batch_run(tvs_batch *batch);
/* Wait and report the first error of the last run. */
int tvs_batch_finish(tvs_batch *batch);
int tvs_batch_read(tvs_batch *batch, uint32_t dem, float *cumulative_out, float *total_out);
void *tvs_batch_stream(const tvs_batch *batch);
uint64_t tvs_batch_device_bytes(const tvs_batch *batch);

/* ---- allocation-free form -------------------------------------------- */

/* No counterpart in the reference.  One sector for callers that cannot
 * allocate device memory when they call: hosts whose device memory belongs to
 * another allocator (a framework's caching allocator or a fixed pool that must
 * account for every byte), and real-time callers that forbid allocation after
 * start-up because an allocation can block or fail at any moment.  Inputs and outputs are the caller's device pointers: d_elevations
 * (width*height f32), d_cumulative (in/out) and d_total (in/out, nullable),
 * computable_points_count f32 each, on device params->device (the call makes
 * that device current and restores the caller's current device before it
 * returns).  The sector's intermediate tables live in
 * a 64 KiB static device array inside the library (held by every GPU that
 * loads it, until exit); lines of sight longer than ~1590 cells do not fit and
 * return TVS_ERR_CAPACITY.  Exact f32 only.  The call is synchronous on
 * `stream` (a cudaStream_t of that device, NULL for the legacy stream).  All calls share the
 * array and overlapping calls would race: the library serialises its own
 * calls.  The first call on a device looks up the array's device address:
 * make it before any stream capture.  Error text: tvs_last_error(NULL). */
int tvs_compute_sector_noalloc(const tvs_params *params, const float *d_elevations,
                               uint32_t angle, float *d_cumulative, float *d_total,
                               void *stream);

/* ---- self-checks ------------------------------------------------------ */

/* Compare the sweep's table-driven division with CUDA's IEEE division
 * (__fdiv_rn) on n pseudo-random (numerator, distance) pairs drawn from
 * seed; returns the number of bitwise mismatches in *mismatches. */
int tvs_selftest_division(int32_t device, uint64_t n, uint64_t seed, uint64_t *mismatches);

/* FP32 issue-rate microbenchmark (independent FFMA chains on every SM):
 * measured FP32 lane-instructions per second, the sweep's roofline peak. */
int tvs_measure_fp32_issue(int32_t device, double *instructions_per_second);

/* L1 load-throughput microbenchmark (every warp loading 32 consecutive
 * floats, the sweep's access, from L1-resident data on every SM): bytes per
 * second, the sweep's secondary roofline peak. */
int tvs_measure_l1_load(int32_t device, double *bytes_per_second);

#ifdef __cplusplus
}
#endif
#endif
