/*
 * tvs_oracle.c -- CPU restatement of the reference total-viewshed hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): see tvs_oracle.h.  Compiled with
 * -ffp-contract=off and without -ffast-math so that every float/double
 * operation is one IEEE-754 round-to-nearest operation, as in the Rust
 * reference (which never contracts to FMA).
 */
#include "tvs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* axes.rs:47 */
static const float SECTOR_SHIFT = 0.001f;
/* axes.rs:35 */
static const uint32_t SECTOR_STEPS = 180;
/* kernel.rs:13 */
static const float MAX_ANGLE = -2000.0f;
/* kernel.rs:17 */
static const float TAN_ONE_RAD = 0.0174533f;
/* kernel.rs:21 (numerically the earth's diameter in metres) */
static const float EARTH_RADIUS_SQUARED = 12742000.0f;
/* Rust `f64::to_radians`: self * (PI / 180.0), the constant folded in f64. */
static const double RADS_PER_DEG = 3.14159265358979323846 / 180.0;
/* band_of_sight.rs:50 core::f64::consts::SQRT_2 */
static const double DIAGONAL_GREATER_THAN_WIDTH = 1.41421356237309504880;

/* Rust `f32 as u32` saturates (NaN -> 0). */
static uint32_t f32_as_u32(float v) {
    if (!(v > 0.0f)) return 0;
    if (v >= 4294967296.0f) return UINT32_MAX;
    return (uint32_t)v;
}

static uint64_t isqrt_u64(uint64_t n) {
    uint64_t r = (uint64_t)sqrt((double)n);
    while (r * r > n) r--;
    while ((r + 1) * (r + 1) <= n) r++;
    return r;
}

/* dem.rs:106-115 is_point_computable, one axis at a time (the test is
 * separable: x and y use the same bounds for a square DEM). */
static uint32_t computable_along(uint32_t extent, float scale, uint32_t los_m) {
    float lower = (float)los_m;
    float upper = ((float)(extent - 1) * scale) - lower;
    uint32_t count = 0;
    for (uint32_t i = 0; i < extent; i++) {
        float v = (float)i * scale;
        if (v >= lower && v <= upper) count++;
    }
    return count;
}

int tvso_geometry_new(uint32_t width, uint32_t height, float scale,
                      uint32_t max_line_of_sight, float rings_per_km,
                      tvso_geometry *out) {
    if (!out || width == 0 || height == 0) return TVSO_ERR_ARGS;
    memset(out, 0, sizeof(*out));
    out->width = width;
    out->height = height;
    out->scale = scale;
    out->max_line_of_sight = max_line_of_sight;
    out->size = (uint64_t)width * height;
    /* dem.rs:53 */
    out->max_los_as_points = f32_as_u32((float)max_line_of_sight / scale);
    /* dem.rs:54-62 (the extension also bounds the height) */
    uint32_t shorter = width < height ? width : height;
    if (out->max_los_as_points > shorter / 2) return TVSO_ERR_LOS_TOO_LONG;
    out->band_size = out->max_los_as_points + 1;
    out->band_deltas_size = out->band_size - 1;
    uint32_t nx = computable_along(width, scale, max_line_of_sight);
    uint32_t ny = computable_along(height, scale, max_line_of_sight);
    out->computable_points_count = (uint64_t)nx * ny;
    if (width == height) {
        /* dem.rs:82 */
        out->tvs_width = (uint32_t)isqrt_u64(out->computable_points_count);
        out->tvs_height = out->tvs_width;
    } else {
        out->tvs_width = nx;
        out->tvs_height = ny;
    }
    out->total_bands = out->computable_points_count * 2;
    /* compute.rs:94-98 */
    float band_length_in_km = (float)max_line_of_sight / 1000.0f;
    out->reserved_rings_per_band = f32_as_u32(band_length_in_km * rings_per_km);
    return TVSO_OK;
}

/* axes.rs:154-176 */
void tvso_calculate_distances(uint32_t width, uint32_t height, float angle, double *out) {
    double angle_f64 = (double)angle;
    double s = sin(angle_f64 * RADS_PER_DEG);
    double c = cos(angle_f64 * RADS_PER_DEG);
    uint64_t k = 0;
    for (int64_t row = 0; row < (int64_t)height; row++) {
        double y = (double)(-row); /* y runs 0, -1, ..., -(H-1); +0.0 first */
        double right = y * c;
        for (uint32_t x = 0; x < width; x++) {
            double left = (double)x * s;
            out[k++] = left - right;
        }
    }
}

/* radsort 0.1.1's f32 key: an order-preserving map to u32 giving the total
 * order -NaN < -inf < ... < -0.0 < +0.0 < ... < +inf < +NaN. */
static inline uint32_t f32_radix_key(float f) {
    uint32_t bits;
    memcpy(&bits, &f, 4);
    uint32_t mask = (uint32_t)(-(int32_t)(bits >> 31)) | 0x80000000u;
    return bits ^ mask;
}

/* Stable LSD radix sort of ids by key, 8-bit digits (radsort's method):
 * the result equals a sort on (key, id). */
static int radix_order(const uint32_t *keys_in, uint64_t n, uint32_t *order_out) {
    uint32_t *ka = malloc(n * sizeof(uint32_t));
    uint32_t *kb = malloc(n * sizeof(uint32_t));
    uint32_t *ib = malloc(n * sizeof(uint32_t));
    if (!ka || !kb || !ib) {
        free(ka); free(kb); free(ib);
        return TVSO_ERR_NOMEM;
    }
    memcpy(ka, keys_in, n * sizeof(uint32_t));
    uint32_t *ia = order_out;
    for (uint64_t i = 0; i < n; i++) ia[i] = (uint32_t)i;
    for (int pass = 0; pass < 4; pass++) {
        int shift = pass * 8;
        uint64_t count[257];
        memset(count, 0, sizeof(count));
        for (uint64_t i = 0; i < n; i++) count[((ka[i] >> shift) & 0xFFu) + 1]++;
        for (int b = 0; b < 256; b++) count[b + 1] += count[b];
        for (uint64_t i = 0; i < n; i++) {
            uint32_t d = (ka[i] >> shift) & 0xFFu;
            uint64_t p = count[d]++;
            kb[p] = ka[i];
            ib[p] = ia[i];
        }
        uint32_t *t = ka; ka = kb; kb = t;
        t = ia; ia = ib; ib = t;
    }
    /* four passes: the sorted ids are back in order_out (ia == order_out). */
    free(ka); free(kb); free(ib);
    return TVSO_OK;
}

/* axes.rs:70-85 */
int tvso_order_by_distance(const double *distances, uint64_t n, uint32_t *order_out) {
    uint32_t *keys = malloc(n * sizeof(uint32_t));
    if (!keys) return TVSO_ERR_NOMEM;
    for (uint64_t i = 0; i < n; i++) keys[i] = f32_radix_key((float)distances[i]);
    int rc = radix_order(keys, n, order_out);
    free(keys);
    return rc;
}

/* Axes::new + Axes::compute (axes.rs:89-130).  Internal form that keeps the
 * sight_ordered_map (rank of every id) the shape stage needs. */
static int axes_compute(uint32_t width, uint32_t height, float angle, float *distances32,
                        uint32_t *sight_rank_of_id, uint32_t *sight_order,
                        uint32_t *sector_ordered) {
    uint64_t n = (uint64_t)width * height;
    float shifted = angle + SECTOR_SHIFT;              /* axes.rs:95 (f32) */
    double *d = malloc(n * sizeof(double));
    uint32_t *order = malloc(n * sizeof(uint32_t));
    if (!d || !order) { free(d); free(order); return TVSO_ERR_NOMEM; }
    int rc;
    tvso_calculate_distances(width, height, shifted, d);
    rc = tvso_order_by_distance(d, n, order);
    if (rc) goto done;
    if (distances32)
        for (uint64_t i = 0; i < n; i++) distances32[i] = (float)d[i];
    if (sight_rank_of_id)
        for (uint64_t r = 0; r < n; r++) sight_rank_of_id[order[r]] = (uint32_t)r;
    if (sight_order) memcpy(sight_order, order, n * sizeof(uint32_t));
    if (sector_ordered) {
        tvso_calculate_distances(width, height, shifted + 90.0f, d);  /* axes.rs:127 */
        rc = tvso_order_by_distance(d, n, sector_ordered);
    }
done:
    free(d);
    free(order);
    return rc;
}

int tvso_axes(uint32_t width, uint32_t height, float angle, float *distances,
              uint32_t *sight_order, uint32_t *sector_ordered) {
    if (width == 0 || height == 0) return TVSO_ERR_ARGS;
    return axes_compute(width, height, angle, distances, NULL, sight_order, sector_ordered);
}

typedef struct { uint32_t rank; uint32_t pos; } rank_pos;

static int cmp_rank_pos(const void *a, const void *b) {
    uint32_t x = ((const rank_pos *)a)->rank, y = ((const rank_pos *)b)->rank;
    return (x > y) - (x < y);
}

/* The square the band shape is built on: the whole DEM when it is square (the
 * reference), the central min(W, H) square of a rectangular DEM (the
 * extension: the reference's construction on the long axis of an elongated
 * DEM makes strip steps long enough to leave it). */
static void shape_window(const tvso_geometry *g, uint32_t *side, uint32_t *x0, uint32_t *y0) {
    uint32_t s = g->width < g->height ? g->width : g->height;
    *side = s;
    *x0 = (g->width - s) / 2;
    *y0 = (g->height - s) / 2;
}

/* axes.rs:154-176 for one point given by its DEM id. */
static double projection_of(uint32_t width, uint64_t id, double s, double c) {
    double y = (double)(-(int64_t)(id / width));
    double right = y * c;
    double left = (double)(id % width) * s;
    return left - right;
}

/* band_of_sight.rs:61-174 */
int tvso_compile_band_data(const tvso_geometry *g, float angle, int32_t *deltas,
                           float *dists, uint32_t *n_filled) {
    if (!g || !deltas || !dists) return TVSO_ERR_ARGS;
    uint32_t side, x0, y0;
    shape_window(g, &side, &x0, &y0);
    const uint64_t n = (uint64_t)side * side;           /* points of the window */
    const float shifted = angle + SECTOR_SHIFT;         /* axes.rs:95 (f32) */
    const double ss = sin((double)shifted * RADS_PER_DEG), sc = cos((double)shifted * RADS_PER_DEG);
    const float sector_angle = shifted + 90.0f;         /* axes.rs:127 */
    const double ts = sin((double)sector_angle * RADS_PER_DEG);
    const double tc = cos((double)sector_angle * RADS_PER_DEG);
    double *d = malloc(n * sizeof(double));
    uint32_t *ids = malloc(n * sizeof(uint32_t));       /* local index -> DEM id */
    uint32_t *order = malloc(n * sizeof(uint32_t));
    uint32_t *rank = malloc(n * sizeof(uint32_t));      /* local index -> sight rank */
    uint32_t *sector = malloc(n * sizeof(uint32_t));    /* sector rank -> local index */
    rank_pos *window = NULL;
    uint32_t *window_ids = NULL;
    int rc = TVSO_ERR_NOMEM;
    if (!d || !ids || !order || !rank || !sector) goto done;
    /* window points in row-major order (ascending DEM id), as axes.rs:160-172
     * enumerates a square DEM */
    for (uint64_t k = 0; k < n; k++)
        ids[k] = (uint32_t)((uint64_t)(y0 + k / side) * g->width + x0 + k % side);
    for (uint64_t k = 0; k < n; k++) d[k] = projection_of(g->width, ids[k], ss, sc);
    rc = tvso_order_by_distance(d, n, order);
    if (rc) goto done;
    for (uint64_t r = 0; r < n; r++) rank[order[r]] = (uint32_t)r;
    for (uint64_t k = 0; k < n; k++) d[k] = projection_of(g->width, ids[k], ts, tc);
    rc = tvso_order_by_distance(d, n, sector);
    if (rc) goto done;

    uint32_t dsize = g->band_deltas_size;
    memset(deltas, 0, dsize * sizeof(int32_t));           /* :67 */
    memset(dists, 0, dsize * sizeof(float));              /* :68 */

    /* :95 (f64 product truncated to usize) */
    uint64_t band_samples =
        (uint64_t)((double)(g->band_size * 2) * DIAGONAL_GREATER_THAN_WIDTH);
    uint64_t pov_local = n / 2;                           /* :99 */
    rc = TVSO_ERR_SHAPE_PANIC;
    if (band_samples / 2 > pov_local) goto done;          /* :103 usize underflow */
    uint64_t band_edge = pov_local - band_samples / 2;
    if (band_edge + band_samples > n) goto done;          /* :113 index */

    window = malloc(band_samples * sizeof(rank_pos));
    window_ids = malloc(band_samples * sizeof(uint32_t));
    rc = TVSO_ERR_NOMEM;
    if (!window || !window_ids) goto done;
    for (uint64_t i = 0; i < band_samples; i++) {         /* :111-120 */
        uint32_t local = sector[band_edge + i];
        window_ids[i] = ids[local];
        window[i].rank = rank[local];
        window[i].pos = (uint32_t)i;
    }
    /* :135-145 ranks are unique, so any sort gives the same permutation */
    qsort(window, band_samples, sizeof(rank_pos), cmp_rank_pos);

    uint64_t middle = band_samples / 2;                   /* :149 */
    uint64_t end_of_band = (uint64_t)g->band_size * 2;    /* :150 */
    float pov_distance = (float)projection_of(g->width, ids[pov_local], ss, sc);  /* :157 */
    uint32_t filled = 0;
    rc = TVSO_ERR_SHAPE_PANIC;
    for (uint64_t band_id = middle; band_id < end_of_band; band_id++) {
        uint64_t i = band_id - middle;
        if (band_id + 1 >= band_samples) goto done;       /* :162 index */
        if (i >= dsize) goto done;                        /* :165 index */
        int32_t current = (int32_t)window_ids[window[band_id].pos];
        int32_t next = (int32_t)window_ids[window[band_id + 1].pos];
        deltas[i] = current - next;                       /* :164 */
        float next_distance = (float)projection_of(g->width, (uint32_t)next, ss, sc);
        dists[i] = fabsf(pov_distance - next_distance);   /* :167-168 */
        filled++;
    }
    if (n_filled) *n_filled = filled;
    rc = TVSO_OK;
done:
    free(d); free(ids); free(order); free(rank); free(sector); free(window); free(window_ids);
    return rc;
}

/* One band's result: its surface and the ring ids in write order. */
typedef struct {
    int status;
    uint32_t n_ids;      /* ring_id at the end == ids written after slot 0 */
    uint32_t *ids;       /* ids[0] = pov, then open/close events */
} band_out;

/* kernel.rs:71-256 for one band (kernel_id), f32 arithmetic. */
static float sweep_band_f32(const tvso_geometry *g, uint64_t kernel_id,
                            const float *elev, float observer_height,
                            const int32_t *deltas, const float *dists,
                            band_out *o) {
    uint64_t half_total_bands = g->total_bands / 2;
    int forward = kernel_id < half_total_bands;
    uint64_t tvs_id = forward ? kernel_id : kernel_id - half_total_bands;
    uint64_t pov_x = tvs_id % g->tvs_width + g->max_los_as_points;
    uint64_t pov_y = tvs_id / g->tvs_width + g->max_los_as_points;
    int64_t pov_id = (int64_t)(pov_y * g->width + pov_x);
    float pov_elevation = elev[pov_id] + observer_height;     /* :134 */
    float max_angle = MAX_ANGLE;
    int is_currently_visible = 1, closing = 0, is_previously_visible = 1;
    float band_surface = 0.0f;
    uint32_t ring_id = 1;
    o->ids[0] = (uint32_t)pov_id;                              /* :145 */
    int64_t dem_id = pov_id;
    o->status = TVSO_OK;
    for (uint32_t i = 0; i < g->band_deltas_size; i++) {
        int32_t delta = deltas[i];
        dem_id = forward ? dem_id + delta : dem_id - delta;    /* :157-160 */
        if (dem_id < 0 || (uint64_t)dem_id >= g->size) {
            o->status = TVSO_ERR_ELEVATION_OOB;
            o->n_ids = ring_id;
            return band_surface;
        }
        float elevation_delta = elev[dem_id] - pov_elevation;  /* :164 */
        float distance = dists[i];
        float angle = (elevation_delta / distance) - (distance / EARTH_RADIUS_SQUARED);
        is_currently_visible = angle > max_angle;              /* :190 */
        int opening = is_currently_visible && !is_previously_visible;
        closing = is_previously_visible && !is_currently_visible;
        if (is_currently_visible) band_surface += distance * TAN_ONE_RAD;
        if (opening) o->ids[ring_id++] = (uint32_t)dem_id;
        if (closing) o->ids[ring_id++] = (uint32_t)dem_id;
        is_previously_visible = is_currently_visible;
        max_angle = fmaxf(angle, max_angle);                   /* :233 f32::max */
    }
    if (is_currently_visible && !closing) o->ids[ring_id++] = (uint32_t)dem_id;
    o->n_ids = ring_id;
    return band_surface;
}

/* The same control flow in double precision. */
static double sweep_band_f64(const tvso_geometry *g, uint64_t kernel_id,
                             const float *elev, float observer_height,
                             const int32_t *deltas, const float *dists,
                             band_out *o) {
    uint64_t half_total_bands = g->total_bands / 2;
    int forward = kernel_id < half_total_bands;
    uint64_t tvs_id = forward ? kernel_id : kernel_id - half_total_bands;
    uint64_t pov_x = tvs_id % g->tvs_width + g->max_los_as_points;
    uint64_t pov_y = tvs_id / g->tvs_width + g->max_los_as_points;
    int64_t pov_id = (int64_t)(pov_y * g->width + pov_x);
    double pov_elevation = (double)elev[pov_id] + (double)observer_height;
    double max_angle = -2000.0;
    int is_currently_visible = 1, closing = 0, is_previously_visible = 1;
    double band_surface = 0.0;
    uint32_t ring_id = 1;
    o->ids[0] = (uint32_t)pov_id;
    int64_t dem_id = pov_id;
    o->status = TVSO_OK;
    for (uint32_t i = 0; i < g->band_deltas_size; i++) {
        int32_t delta = deltas[i];
        dem_id = forward ? dem_id + delta : dem_id - delta;
        if (dem_id < 0 || (uint64_t)dem_id >= g->size) {
            o->status = TVSO_ERR_ELEVATION_OOB;
            o->n_ids = ring_id;
            return band_surface;
        }
        double elevation_delta = (double)elev[dem_id] - pov_elevation;
        double distance = (double)dists[i];
        double angle = (elevation_delta / distance) - (distance / 12742000.0);
        is_currently_visible = angle > max_angle;
        int opening = is_currently_visible && !is_previously_visible;
        closing = is_previously_visible && !is_currently_visible;
        if (is_currently_visible) band_surface += distance * 0.0174533;
        if (opening) o->ids[ring_id++] = (uint32_t)dem_id;
        if (closing) o->ids[ring_id++] = (uint32_t)dem_id;
        is_previously_visible = is_currently_visible;
        max_angle = fmax(angle, max_angle);
    }
    if (is_currently_visible && !closing) o->ids[ring_id++] = (uint32_t)dem_id;
    o->n_ids = ring_id;
    return band_surface;
}

/* The plain reciprocal-table FP32 form of kernel.rs:175 (the comparison
 * baseline of the engine, not the reference's arithmetic): per step the tables
 * y = RN(1/d), c = RN(d/12742000) and w = RN(d*0.0174533f) in f32, the angle
 * fmaf(RN(h - h_pov), y, -c) (one rounding), f32 comparisons and f32 surface
 * sums.  The control flow and the ring records are kernel.rs:153-243's. */
static float sweep_band_fp32(const tvso_geometry *g, uint64_t kernel_id,
                             const float *elev, float observer_height,
                             const int32_t *deltas, const float *dists,
                             band_out *o) {
    uint64_t half_total_bands = g->total_bands / 2;
    int forward = kernel_id < half_total_bands;
    uint64_t tvs_id = forward ? kernel_id : kernel_id - half_total_bands;
    uint64_t pov_x = tvs_id % g->tvs_width + g->max_los_as_points;
    uint64_t pov_y = tvs_id / g->tvs_width + g->max_los_as_points;
    int64_t pov_id = (int64_t)(pov_y * g->width + pov_x);
    float pov_elevation = elev[pov_id] + observer_height;
    float max_angle = MAX_ANGLE;
    int is_currently_visible = 1, closing = 0, is_previously_visible = 1;
    float band_surface = 0.0f;
    uint32_t ring_id = 1;
    o->ids[0] = (uint32_t)pov_id;
    int64_t dem_id = pov_id;
    o->status = TVSO_OK;
    for (uint32_t i = 0; i < g->band_deltas_size; i++) {
        int32_t delta = deltas[i];
        dem_id = forward ? dem_id + delta : dem_id - delta;
        if (dem_id < 0 || (uint64_t)dem_id >= g->size) {
            o->status = TVSO_ERR_ELEVATION_OOB;
            o->n_ids = ring_id;
            return band_surface;
        }
        float distance = dists[i];
        float y = 1.0f / distance;
        float c = distance / EARTH_RADIUS_SQUARED;
        float angle = fmaf(elev[dem_id] - pov_elevation, y, -c);
        is_currently_visible = angle > max_angle;
        int opening = is_currently_visible && !is_previously_visible;
        closing = is_previously_visible && !is_currently_visible;
        if (is_currently_visible) band_surface += distance * TAN_ONE_RAD;
        if (opening) o->ids[ring_id++] = (uint32_t)dem_id;
        if (closing) o->ids[ring_id++] = (uint32_t)dem_id;
        is_previously_visible = is_currently_visible;
        max_angle = fmaxf(angle, max_angle);
    }
    if (is_currently_visible && !closing) o->ids[ring_id++] = (uint32_t)dem_id;
    o->n_ids = ring_id;
    return band_surface;
}

/* kernel.rs:141-145,220-243,302-309: replay one band's ring writes into the
 * flat sector buffer in the reference's order (slot 1 .. n, then slot 0).
 * An index past the buffer is the reference's out-of-bounds panic. */
static int save_band_rings(uint64_t kernel_id, uint32_t reserved, const band_out *o,
                           uint32_t *rings, uint64_t rings_len) {
    uint64_t start = kernel_id * (uint64_t)reserved;
    for (uint32_t j = 1; j <= o->n_ids; j++) {
        uint64_t at = start + j;
        if (at >= rings_len) return TVSO_ERR_RING_OOB;
        rings[at] = o->ids[j - 1];
    }
    if (start >= rings_len) return TVSO_ERR_RING_OOB;
    rings[start] = o->n_ids;
    return TVSO_OK;
}

/* One sector over the bands of computable rows [o->row_begin, o->row_end)
 * (all rows when both are 0), forward bands before backward bands as
 * compute.rs:229 orders them.  Surfaces go to o->cum32 / o->cum64 indexed from
 * the first row of the range; ring records to the reference layout and/or the
 * compact stream. */
static int compute_sector_impl(const tvso_geometry *g, const float *elev,
                               float observer_height, const int32_t *deltas,
                               const float *dists, const tvso_sweep_opts *opt) {
    if (!g || !elev || !deltas || !dists || !opt) return TVSO_ERR_ARGS;
    uint32_t rb = opt->row_begin, re = opt->row_end;
    if (rb == 0 && re == 0) re = g->tvs_height;
    if (rb > re || re > g->tvs_height) return TVSO_ERR_ARGS;
    const int mode = opt->mode;
    if (mode < TVSO_MODE_EXACT32 || mode > TVSO_MODE_FP32) return TVSO_ERR_ARGS;
    const int f64 = mode == TVSO_MODE_F64;
    if (f64 ? !opt->cum64 : !opt->cum32) return TVSO_ERR_ARGS;
    uint64_t half = g->total_bands / 2;
    uint64_t t0 = (uint64_t)rb * g->tvs_width, t1 = (uint64_t)re * g->tvs_width;
    uint64_t local = t1 - t0;
    uint32_t max_ids = g->band_deltas_size + 2;
    /* Per tvs id of the range: forward and backward surfaces and ring ids. */
    float *sf32 = NULL, *sb32 = NULL;
    double *sf64 = NULL, *sb64 = NULL;
    band_out *outs = NULL;
    uint32_t *id_store = NULL;
    uint64_t n_ids_total = 0;
    int rc = TVSO_ERR_NOMEM;
    if (opt->counts) memset(opt->counts, 0, g->total_bands * sizeof(uint32_t));
    if (!f64) {
        sf32 = malloc((local ? local : 1) * sizeof(float));
        sb32 = malloc((local ? local : 1) * sizeof(float));
        if (!sf32 || !sb32) goto done;
    } else {
        sf64 = malloc((local ? local : 1) * sizeof(double));
        sb64 = malloc((local ? local : 1) * sizeof(double));
        if (!sf64 || !sb64) goto done;
    }
    /* Bands are processed in blocks so the ring-id store stays bounded. */
    const uint64_t block = 4096;
    outs = malloc(2 * block * sizeof(band_out));
    id_store = malloc(2 * block * (uint64_t)max_ids * sizeof(uint32_t));
    if (!outs || !id_store) goto done;
    for (uint64_t j = 0; j < 2 * block; j++) outs[j].ids = id_store + j * max_ids;
#ifdef _OPENMP
    int threads = opt->threads < 1 ? 1 : opt->threads;
    omp_set_num_threads(threads);
#endif
    rc = TVSO_OK;
    /* Forward bands (kernel ids 0..half) all run before the backward bands
     * (compute.rs:229): surfaces are added in that order below, and the ring
     * writes are replayed in kernel-id order. */
    for (int dir = 0; dir < 2 && rc == TVSO_OK; dir++) {
        for (uint64_t b0 = t0; b0 < t1 && rc == TVSO_OK; b0 += block) {
            uint64_t nb = t1 - b0 < block ? t1 - b0 : block;
#pragma omp parallel for schedule(static)
            for (int64_t j = 0; j < (int64_t)nb; j++) {
                uint64_t tvs = b0 + (uint64_t)j;
                uint64_t kid = dir == 0 ? tvs : tvs + half;
                band_out *o = &outs[j];
                if (f64) {
                    double sv = sweep_band_f64(g, kid, elev, observer_height, deltas, dists, o);
                    (dir == 0 ? sf64 : sb64)[tvs - t0] = sv;
                } else {
                    float sv = mode == TVSO_MODE_FP32
                                   ? sweep_band_fp32(g, kid, elev, observer_height, deltas, dists, o)
                                   : sweep_band_f32(g, kid, elev, observer_height, deltas, dists, o);
                    (dir == 0 ? sf32 : sb32)[tvs - t0] = sv;
                }
            }
            for (uint64_t j = 0; j < nb; j++) {
                uint64_t tvs = b0 + j;
                uint64_t kid = dir == 0 ? tvs : tvs + half;
                if (outs[j].status != TVSO_OK) { rc = outs[j].status; break; }
                if (opt->rings) {
                    int r = save_band_rings(kid, g->reserved_rings_per_band, &outs[j],
                                            opt->rings, opt->rings_len);
                    if (r != TVSO_OK) { rc = r; break; }
                }
                if (opt->counts) {
                    /* ids past ids_cap are counted, not copied: *ids_total > ids_cap
                     * tells the caller that the stream was cut */
                    opt->counts[kid] = outs[j].n_ids;
                    if (opt->ids && n_ids_total + outs[j].n_ids <= opt->ids_cap)
                        memcpy(opt->ids + n_ids_total, outs[j].ids, outs[j].n_ids * sizeof(uint32_t));
                    n_ids_total += outs[j].n_ids;
                }
            }
        }
    }
    if (rc != TVSO_OK) goto done;
    if (opt->ids_total) *opt->ids_total = n_ids_total;
    /* kernel.rs:254: cumulative[tvs] += surface, forward band first. */
    for (uint64_t t = 0; t < local; t++) {
        if (!f64) {
            opt->cum32[t] += sf32[t];
            opt->cum32[t] += sb32[t];
        } else {
            opt->cum64[t] += sf64[t];
            opt->cum64[t] += sb64[t];
        }
    }
done:
    free(sf32); free(sb32); free(sf64); free(sb64); free(outs); free(id_store);
    return rc;
}

int tvso_sweep_sector(const tvso_geometry *g, const float *elevations, float observer_height,
                      const int32_t *deltas, const float *dists, const tvso_sweep_opts *opts) {
    return compute_sector_impl(g, elevations, observer_height, deltas, dists, opts);
}

int tvso_compute_sector(const tvso_geometry *g, const float *elevations,
                        float observer_height, const int32_t *deltas,
                        const float *dists, float *cumulative, uint32_t *rings,
                        uint64_t rings_len, int threads) {
    if (!cumulative) return TVSO_ERR_ARGS;
    tvso_sweep_opts o = {0};
    o.mode = TVSO_MODE_EXACT32;
    o.cum32 = cumulative;
    o.rings = rings;
    o.rings_len = rings_len;
    o.threads = threads;
    return compute_sector_impl(g, elevations, observer_height, deltas, dists, &o);
}

int tvso_compute_sector_f64(const tvso_geometry *g, const float *elevations,
                            float observer_height, const int32_t *deltas,
                            const float *dists, double *cumulative,
                            uint32_t *rings, uint64_t rings_len, int threads) {
    if (!cumulative) return TVSO_ERR_ARGS;
    tvso_sweep_opts o = {0};
    o.mode = TVSO_MODE_F64;
    o.cum64 = cumulative;
    o.rings = rings;
    o.rings_len = rings_len;
    o.threads = threads;
    return compute_sector_impl(g, elevations, observer_height, deltas, dists, &o);
}

static int run_impl(const tvso_geometry *g, const float *elev, float observer_height,
                    uint32_t first_angle, uint32_t n_angles, int mode, uint32_t rb, uint32_t re,
                    float *cum32, float *total, double *cum64, uint32_t *rings_all,
                    int threads) {
    if (!g || !elev || first_angle + n_angles > SECTOR_STEPS) return TVSO_ERR_ARGS;
    if (rb == 0 && re == 0) re = g->tvs_height;
    if (rb > re || re > g->tvs_height) return TVSO_ERR_ARGS;
    uint64_t count = (uint64_t)(re - rb) * g->tvs_width;
    uint64_t ring_len = g->total_bands * (uint64_t)g->reserved_rings_per_band;
    int32_t *deltas = calloc(g->band_deltas_size ? g->band_deltas_size : 1, sizeof(int32_t));
    float *dists = calloc(g->band_deltas_size ? g->band_deltas_size : 1, sizeof(float));
    if (!deltas || !dists) { free(deltas); free(dists); return TVSO_ERR_NOMEM; }
    if (cum32) memset(cum32, 0, count * sizeof(float));      /* compute.rs:102 */
    if (cum64) memset(cum64, 0, count * sizeof(double));
    if (total) memset(total, 0, count * sizeof(float));      /* compute.rs:103 */
    if (rings_all) memset(rings_all, 0, (uint64_t)n_angles * ring_len * sizeof(uint32_t));
    int rc = TVSO_OK;
    for (uint32_t a = 0; a < n_angles && rc == TVSO_OK; a++) {
        uint32_t angle = first_angle + a;
        rc = tvso_compile_band_data(g, (float)angle, deltas, dists, NULL);
        if (rc) break;
        tvso_sweep_opts o = {0};
        o.mode = mode;
        o.row_begin = rb;
        o.row_end = re;
        o.cum32 = cum32;
        o.cum64 = cum64;
        o.rings = rings_all ? rings_all + (uint64_t)a * ring_len : NULL;
        o.rings_len = ring_len;
        o.threads = threads;
        rc = compute_sector_impl(g, elev, observer_height, deltas, dists, &o);
        if (rc) break;
        if (total && cum32)                                  /* compute.rs:206-214 */
            for (uint64_t t = 0; t < count; t++) total[t] += cum32[t];
    }
    free(deltas);
    free(dists);
    return rc;
}

int tvso_run(const tvso_geometry *g, const float *elevations, float observer_height,
             uint32_t first_angle, uint32_t n_angles, float *cumulative,
             float *total, uint32_t *rings_all, int threads) {
    if (!cumulative) return TVSO_ERR_ARGS;
    return run_impl(g, elevations, observer_height, first_angle, n_angles, TVSO_MODE_EXACT32,
                    0, 0, cumulative, total, NULL, rings_all, threads);
}

int tvso_run_f64(const tvso_geometry *g, const float *elevations,
                 float observer_height, uint32_t first_angle, uint32_t n_angles,
                 double *cumulative, uint32_t *rings_all, int threads) {
    if (!cumulative) return TVSO_ERR_ARGS;
    return run_impl(g, elevations, observer_height, first_angle, n_angles, TVSO_MODE_F64,
                    0, 0, NULL, NULL, cumulative, rings_all, threads);
}

int tvso_run_ex(const tvso_geometry *g, const float *elevations, float observer_height,
                uint32_t first_angle, uint32_t n_angles, int mode, uint32_t row_begin,
                uint32_t row_end, float *cumulative32, float *total, double *cumulative64,
                int threads) {
    if (mode == TVSO_MODE_F64 ? !cumulative64 : !cumulative32) return TVSO_ERR_ARGS;
    return run_impl(g, elevations, observer_height, first_angle, n_angles, mode, row_begin,
                    row_end, mode == TVSO_MODE_F64 ? NULL : cumulative32,
                    mode == TVSO_MODE_F64 ? NULL : total,
                    mode == TVSO_MODE_F64 ? cumulative64 : NULL, NULL, threads);
}
