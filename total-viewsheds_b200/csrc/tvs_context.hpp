// tvs_context.hpp -- the per-DEM context behind the C ABI (internal to the library).
#pragma once

#include <cstdint>
#include <string>

#include "tvs.h"
#include "tvs_internal.cuh"

struct tvs_context {
    tvs_params p{};
    tvs_geometry g{};
    uint32_t row_begin = 0, row_end = 0;
    int64_t pov_min = 0, pov_max = 0;
    uint32_t step_cap = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t launches = 0;

    float *d_elev = nullptr;
    float *d_cum = nullptr;
    float *d_total = nullptr;
    double *d_cum64 = nullptr;
    tvs::SectorTrig *d_trig = nullptr;
    tvs::ShapeHeader *d_hdr = nullptr;   // [180 + 1]: the last slot serves tvs_axes
    float4 *d_steps = nullptr;
    int2 *d_offs = nullptr;
    double4 *d_dtab = nullptr;
    // persistent-sweep work queue
    uint32_t *d_queue = nullptr;
    uint32_t *d_done = nullptr;
    uint32_t done_cap = 0;
    int32_t *d_error = nullptr;
    float *d_hmax = nullptr;  // max |elevation| + |observer height| (estimate windows)
    float *d_bmax = nullptr;  // block maxima of the elevations (segment bounds)
    float4 *d_quad = nullptr; // row-interleaved copies (the quad split layout), nullable
    uint32_t bmax_w = 0, bmax_h = 0;
    unsigned long long *d_rechecks = nullptr;  // MIXED64 FP64 re-decisions
    tvs::QueueDem *d_qdem = nullptr;           // this context as a one-DEM queue
    tvs::QueueConfig qcfg{0, 0, 0, 0, 0};            // sweep configuration (autotuned or default)
    tvs::QueueConfig qcfg_uploaded{0, 0, 0, 0, 0};   // the tiling currently in d_qdem
    uint32_t q_tiles_per_sector = 0;
    uint32_t spin_limit = tvs::kDefaultSpinLimit;  // dependency-wait iteration limit
    uint32_t held_tile = 0xFFFFFFFFu;               // failure-detection test hook
    int32_t *d_deltas = nullptr;
    float *d_dists = nullptr;
    // ring output (allocated on first use)
    uint32_t *d_rings = nullptr;
    uint4 *d_spill = nullptr;
    uint32_t *d_counters = nullptr;
    uint32_t spill_cap = 0;
    uint64_t ring_capacity = 0;                // u32 slots in d_rings
    uint32_t compact_slots = 64;               // slots per band behind the compact stream
    tvs::QueueDem *d_qdem_rings = nullptr;     // this context tiled for the ring sweep
    uint32_t ring_layout = 0;                  // the ring sweep's split layout
    uint32_t q_ring_tiles = 0;
    // plain-kernel scratch (allocated on first use)
    float *d_sf = nullptr, *d_sb = nullptr;
    // band shapes installed as tables (the reference's shape cache), in place of
    // computed ones; allocated on first use
    int32_t *d_tab_deltas = nullptr;
    float *d_tab_dists = nullptr;
    unsigned char *d_installed = nullptr;  // [180]
    bool installed[tvs::kSectorSteps] = {};
    // sectors whose shape slot holds this context's shape with an OK status
    // (the shape depends on the geometry and an installed table only, not on
    // the elevations), so the per-sector calls skip the shape stage
    bool shape_ok[tvs::kSectorSteps] = {};
    // compact ring records of the last tvs_compute_sector_rings (allocated on first use)
    uint64_t *d_rc_blocks = nullptr;   // scanned record-length block sums
    uint64_t *d_rc_offsets = nullptr;  // [total_bands + 1]
    uint32_t *d_rc_ids = nullptr;
    uint64_t rc_ids_cap = 0, rc_total = 0;
    uint64_t rc_records = 0;      // records of the last call (sectors x total_bands)
    uint64_t rc_records_cap = 0;  // records d_rc_offsets and d_rc_blocks hold
    bool rc_valid = false;
    // sweep counters (tvs_set_sweep_counters): [0] warp-steps swept, [1] past
    // the first test, [2] in all, [3] spare
    unsigned long long *d_diag = nullptr;
    bool diag_on = false;
    // the whole-TVS pipeline (tvs_device_run_tvs): one captured graph, and the
    // events it records at the start, after the shape stage and at the end
    cudaGraph_t tvs_graph = nullptr;
    cudaGraphExec_t tvs_exec = nullptr;
    cudaEvent_t ev_begin = nullptr, ev_shaped = nullptr, ev_swept = nullptr;
    uint64_t tvs_graph_launches = 0;  // kernels inside the graph
    // sectors whose shape stage ran since the last tvs_device_finish
    bool pending[tvs::kSectorSteps] = {};
    uint64_t device_bytes = 0;  // everything this context allocated on the device
};

// Helpers capi.cu shares with the other host files of the library.
void tvs_set_create_error(const std::string &msg);
namespace tvs_host {
tvs::ShapeArgs shape_args_of(tvs_context *c, uint32_t first_slot);
tvs::QueueDem queue_dem_of(const tvs_context *c);
int header_status_of(tvs_context *c, uint32_t first, uint32_t count);
int fail_of(tvs_context *c, int code, const std::string &msg);
int enqueue_shape_of(tvs_context *c, uint32_t first, uint32_t count);
void drop_tvs_graph_of(tvs_context *c);
}  // namespace tvs_host
