/*
 * tvs_oracle.h -- CPU restatement of the reference total-viewshed hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine:
 * only the test suite, the smoke check and the CPU-baseline leg of the benchmark
 * load it.  The engine in total-viewsheds_b200/csrc never links, calls or falls
 * back to it.
 *
 * Every function restates one piece of tombh/total-viewsheds (Rust) and cites
 * the file:line it follows (paths relative to the reference repository).
 * Parity is pinned by the reference's own unit-test vectors (axes.rs:216-333,
 * band_of_sight.rs:230-315, cache.rs:87-105, compute.rs:306-416), transcribed
 * into tests/golden/reference_vectors.json by tests/golden/extract_reference_vectors.py.
 *
 * Rectangular DEMs (height != width) are an extension: the reference only
 * reads the header width (main.rs:49, dem.rs:44-46).  With height == width
 * every function below reduces to the reference behaviour.
 */
#ifndef TVS_ORACLE_H
#define TVS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes: the reference panics (or bails) in these situations. */
#define TVSO_OK 0
#define TVSO_ERR_ARGS (-1)
#define TVSO_ERR_LOS_TOO_LONG (-2)       /* dem.rs:56-62 bail!                      */
#define TVSO_ERR_SHAPE_PANIC (-3)        /* band_of_sight.rs index out of bounds    */
#define TVSO_ERR_ELEVATION_OOB (-4)      /* kernel.rs:164 elevations[dem_id] panic  */
#define TVSO_ERR_RING_OOB (-5)           /* kernel.rs:307 ring_data[index] panic    */
#define TVSO_ERR_NOMEM (-6)

/* DEM geometry, as DEM::new (dem.rs:44-72) and Compute::new (compute.rs:27-56)
 * derive it. */
typedef struct tvso_geometry {
    uint32_t width;
    uint32_t height;
    float scale;
    uint32_t max_line_of_sight;       /* metres */
    uint32_t max_los_as_points;       /* dem.rs:53 */
    uint32_t band_size;               /* dem.rs:78: los_pts + 1 */
    uint32_t band_deltas_size;        /* band_of_sight.rs:54-58: band_size - 1 */
    uint32_t tvs_width;               /* dem.rs:82 isqrt(count) == computable columns */
    uint32_t tvs_height;              /* computable rows (== tvs_width when square) */
    uint32_t reserved_rings_per_band; /* compute.rs:94-98 */
    uint64_t size;                    /* width * height */
    uint64_t computable_points_count; /* dem.rs:87-115 */
    uint64_t total_bands;             /* compute.rs:34: 2 * computable */
} tvso_geometry;

int tvso_geometry_new(uint32_t width, uint32_t height, float scale,
                      uint32_t max_line_of_sight, float rings_per_km,
                      tvso_geometry *out);

/* axes.rs:154-176: FP64 x*sin(theta) - y*cos(theta) for every point, row-major. */
void tvso_calculate_distances(uint32_t width, uint32_t height, float angle, double *out);

/* axes.rs:70-85 + radsort 0.1.1: stable radix order of the f32-cast keys.
 * order_out[rank] = point id. */
int tvso_order_by_distance(const double *distances, uint64_t n, uint32_t *order_out);

/* axes.rs:89-130 for a sector angle (degrees, before SECTOR_SHIFT).
 * distances: f32 sight distances [n]; sight_order: ids in sight-rank order [n]
 * (the inverse of sight_ordered_map, as the axes tests extract it);
 * sector_ordered: ids in sector-rank order [n].  Any output may be NULL. */
int tvso_axes(uint32_t width, uint32_t height, float angle, float *distances,
              uint32_t *sight_order, uint32_t *sector_ordered);

/* band_of_sight.rs:61-174.  deltas/dists have band_deltas_size entries; the
 * ones the reference never fills stay 0.  n_filled (nullable) receives how
 * many were filled. */
int tvso_compile_band_data(const tvso_geometry *g, float angle, int32_t *deltas,
                           float *dists, uint32_t *n_filled);

/* compute.rs:228-240 + kernel.rs:71-256: one sector, every band, in kernel-id
 * order.  cumulative [computable] is read-modify-written.  rings (nullable)
 * has rings_len u32 and must be zeroed by the caller (compute.rs:108).
 * threads > 1 sweeps bands in parallel and then replays the ring writes in
 * band order, which is bit-identical to the sequential loop. */
int tvso_compute_sector(const tvso_geometry *g, const float *elevations,
                        float observer_height, const int32_t *deltas,
                        const float *dists, float *cumulative, uint32_t *rings,
                        uint64_t rings_len, int threads);

/* The all-FP64 variant: the same control flow with double angles, running
 * maximum and surfaces.  Shape tables stay the reference's f32 values. */
int tvso_compute_sector_f64(const tvso_geometry *g, const float *elevations,
                            float observer_height, const int32_t *deltas,
                            const float *dists, double *cumulative,
                            uint32_t *rings, uint64_t rings_len, int threads);

/* Sweep arithmetic of tvso_sweep_sector / tvso_run_ex. */
#define TVSO_MODE_EXACT32 0   /* kernel.rs:164-233 in f32, the reference            */
#define TVSO_MODE_F64 1       /* the same control flow in double                    */
#define TVSO_MODE_FP32 2      /* reciprocal-table f32 form: fmaf(e, RN(1/d), -RN(d/R)) */

typedef struct tvso_sweep_opts {
    int mode;                      /* TVSO_MODE_*                                        */
    uint32_t row_begin, row_end;   /* computable rows [begin, end); 0, 0 = every row     */
    float *cum32;                  /* f32 modes: [rows * tvs_width] read-modify-written  */
    double *cum64;                 /* TVSO_MODE_F64: [rows * tvs_width]                   */
    uint32_t *rings;               /* reference layout (nullable, zeroed by the caller)  */
    uint64_t rings_len;
    uint32_t *counts;              /* compact records (nullable): ids per band, every   */
                                   /* band of the sector (0 outside the row range)       */
    uint32_t *ids;                 /* the bands' ids back to back, kernel-id order      */
    uint64_t ids_cap;              /*   (nullable; needs counts)                          */
    uint64_t *ids_total;           /* total ids of the records (nullable); when it is   */
                                   /* above ids_cap, only the records that fit whole    */
                                   /* before the cap were copied                         */
    int threads;
} tvso_sweep_opts;

/* compute.rs:228-240 + kernel.rs:71-256 for one sector, with the options above. */
int tvso_sweep_sector(const tvso_geometry *g, const float *elevations, float observer_height,
                      const int32_t *deltas, const float *dists, const tvso_sweep_opts *opts);

/* compute.rs:101-115,200-214: sectors first_angle .. first_angle+n_angles-1.
 * cumulative and total (heatmap running total) [computable] are zeroed here.
 * rings_all (nullable) receives n_angles * (total_bands * reserved) u32. */
int tvso_run(const tvso_geometry *g, const float *elevations, float observer_height,
             uint32_t first_angle, uint32_t n_angles, float *cumulative,
             float *total, uint32_t *rings_all, int threads);

int tvso_run_f64(const tvso_geometry *g, const float *elevations,
                 float observer_height, uint32_t first_angle, uint32_t n_angles,
                 double *cumulative, uint32_t *rings_all, int threads);

/* tvso_run over computable rows [row_begin, row_end) (0, 0 = all) in any mode:
 * the surfaces of those rows only ([rows * tvs_width]); cumulative32 and total
 * for the f32 modes, cumulative64 for TVSO_MODE_F64. */
int tvso_run_ex(const tvso_geometry *g, const float *elevations, float observer_height,
                uint32_t first_angle, uint32_t n_angles, int mode, uint32_t row_begin,
                uint32_t row_end, float *cumulative32, float *total, double *cumulative64,
                int threads);

#ifdef __cplusplus
}
#endif
#endif
