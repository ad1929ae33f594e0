// queue_sched.cuh -- the work queue shared by the persistent sweeps
// (sweep_queue.cu: row layouts; sweep_split.cu: direction-split layouts).
//
// The grid is the resident capacity of the GPU.  Each CTA takes the next
// (sector, tile) item from a global counter in sector-major order, re-stages
// its step tables only when the sector or the DEM changes, and keeps every
// point's sectors in order: item (s, T) waits, after its sweep and before its
// surface writes, until tile T's counter of completed sectors reaches s.  The
// wait is bounded (TVS_ERR_TIMEOUT in the error word, the item's writes
// skipped, later waits give up at once).
#pragma once

#include <cstdint>

#include "tvs.h"
#include "tvs_internal.cuh"

namespace tvs {

constexpr int kQueueTileX = 32;
// warps per CTA of the persistent sweeps (one build-wide value: the host tiles
// the grid with it)
#ifndef TVS_QUEUE_WARPS
#define TVS_QUEUE_WARPS 8
#endif
constexpr int kQueueTileY = TVS_QUEUE_WARPS;
constexpr int kQueueThreads = kQueueTileX * kQueueTileY;

// Direction-split layouts 1-9: a warp holds LX columns x 32/LX rows of lanes;
// each lane sweeps four points of view, LX columns apart (layouts 1-3: LX = 8,
// 16, 32), 2 x 2 of them, LX columns and 32/LX rows apart (layouts 4-6), or
// four rows 32/LX apart in one column (layouts 7, 8: LX = 32, 16), so that one
// load of the warp reads whole 128- or 64-byte rows.  Layout 9 (quad) is
// layout 7's tiling with the four rows read as one float4 from the DEM's
// row-interleaved copies: a warp's load is 512 contiguous bytes.
constexpr int kSplitCols = 4;  // points of view per lane
constexpr int kSplitLayouts = 9;
__host__ __device__ constexpr int split_lx(int layout) {
    return layout == 7 || layout == 9 ? 32 : layout == 8 ? 16 : 4 << ((layout - 1) % 3 + 1);
}
__host__ __device__ constexpr int split_ky(int layout) { return layout > 6 ? 4 : layout > 3 ? 2 : 1; }
__host__ __device__ constexpr int split_tile_w(int layout) {
    return kSplitCols / split_ky(layout) * split_lx(layout);
}
__host__ __device__ constexpr int split_tile_h(int layout) {
    return kQueueTileY * (32 / split_lx(layout)) * split_ky(layout);
}

// Segments of the direction-split fast loop: kSegSteps steps whose samples are
// bounded together.  Per segment: the range of the forward DEM offsets (x, y)
// over its steps, the largest and smallest 1/d and the largest first-test
// offset.
#ifndef TVS_SEG_STEPS
#define TVS_SEG_STEPS 32
#endif
constexpr uint32_t kSegSteps = TVS_SEG_STEPS;
static_assert(kSegSteps >= 1 && kSegSteps <= 32,
              "the staging reduces one segment per warp, one step per lane");
struct __align__(16) SegBound {
    int dx0, dx1, dy0, dy1;
    float ymax, ymin, zmax, pad;
};

struct QueueCtl {
    QueueDem dem;           // the current item's DEM (copied from the descriptor array)
    uint32_t item;
    uint32_t dem_index;     // descriptor index of `dem`
    uint32_t sector;        // the staged sector
    uint32_t tile;          // the current item's tile within its DEM
    int32_t sector_status;  // the staged sector's shape status
    int32_t wait_status;    // this item's dependency wait
    uint32_t n_steps;
    uint32_t n_fast;
    bool restage;
    bool plain;             // quad layout: the staged sector reads the plain DEM
    float hmax;             // the staged DEM's elevation range (estimate windows)
    unsigned long long diag[4];  // per-item counters (sweep_split.cu), flushed per item
};

#ifdef __CUDACC__
__device__ __forceinline__ void queue_init(QueueCtl &ctl, uint32_t tid) {
    if (tid == 0) {
        ctl.dem_index = 0xFFFFFFFFu;
        ctl.sector = 0xFFFFFFFFu;
    }
}

// Takes the next item (thread 0) and publishes it to the CTA.  Returns false
// (for the whole CTA) when the queue is empty.
__device__ __forceinline__ bool queue_next(const QueueArgs &a, QueueCtl &ctl, uint32_t tid) {
    const uint32_t n_items = a.tiles_per_sector * a.n_sectors;
    if (tid == 0) {
        const uint32_t item = atomicAdd(a.queue, 1u);
        ctl.item = item;
        if (item < n_items) {
            const uint32_t s = item / a.tiles_per_sector;
            const uint32_t r = item - s * a.tiles_per_sector;
            // the DEM whose tiles hold r (tile_base ascends)
            uint32_t lo = 0, hi = a.n_dems - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (a.dems[mid].tile_base <= r) lo = mid; else hi = mid - 1;
            }
            ctl.restage = lo != ctl.dem_index || s != ctl.sector;
            if (lo != ctl.dem_index) ctl.dem = a.dems[lo];
            ctl.dem_index = lo;
            ctl.sector = s;
            ctl.tile = r - ctl.dem.tile_base;
        }
    }
    __syncthreads();
    return ctl.item < n_items;
}

// The tile's previous sector must be complete before this sector's surfaces
// are added.  Every thread of the CTA calls it; returns whether to write.
__device__ __forceinline__ bool queue_wait_prev(const QueueArgs &a, QueueCtl &ctl,
                                                const QueueDem &D, uint32_t s, uint32_t tile,
                                                uint32_t tid) {
    if (tid == 0) {
        ctl.wait_status = TVS_OK;
        if (s > 0) {
            const volatile uint32_t *d = a.done + D.done_base + tile;
            const volatile int32_t *err = a.error;
            uint32_t spins = 0;
            while (*d < s) {
                // give up at the limit, or at once when another wait already did
                if (++spins > a.spin_limit || *err != 0) {
                    atomicExch(a.error, (int32_t)TVS_ERR_TIMEOUT);
                    ctl.wait_status = TVS_ERR_TIMEOUT;
                    break;
                }
                __nanosleep(256);
            }
            __threadfence();
        }
    }
    __syncthreads();
    return ctl.wait_status == TVS_OK;
}

// This item's writes are done: advance the tile's counter of completed sectors.
__device__ __forceinline__ void queue_done(const QueueArgs &a, const QueueDem &D, uint32_t tile,
                                           uint32_t tid) {
    __threadfence();  // this thread's surface writes before the tile's counter
    __syncthreads();
    if (tid == 0 && D.done_base + tile != a.held_tile) atomicAdd(a.done + D.done_base + tile, 1u);
}
#endif

// Host: grid-wide launch of a persistent queue kernel: the shared-memory
// attribute (only ever raised) and the occupancy are kept per (kernel, device)
// under a lock; the queue and tile counters are reset on the stream first.
cudaError_t launch_persistent(const void *fn, const QueueArgs &a, size_t smem, cudaStream_t s);

}  // namespace tvs
