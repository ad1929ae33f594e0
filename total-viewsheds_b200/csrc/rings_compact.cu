// rings_compact.cu -- one sector's ring records as a compact stream.
//
// The reference keeps `reserved` u32 slots per band of sight (kernel.rs:141-145,
// 220-243, 302-309): [n, pov, closing, opening, closing, ...] with n the number
// of ids after the count.  At 3601^2 that is 2.08 GB per sector, mostly zeros,
// and a band whose ids do not fit spills into the next band's slots.  The
// compact stream keeps every band's n ids back to back: band k's ids are
// ids[offsets[k] .. offsets[k+1]), never truncated.  The ring sweep writes
// the reserved layout on the device (ids past the reserved slots go to a
// spill list); these kernels measure, scan and gather it.
#include "tvs.h"
#include "tvs_internal.cuh"

namespace tvs {
namespace {

constexpr int kRingThreads = 1024;
constexpr int kRingPer = 4;                          // bands per thread
constexpr int kRingChunk = kRingThreads * kRingPer;  // bands per CTA
static_assert(kRingThreads == 1024, "block_exclusive scans 32 warp sums in one warp");

// Exclusive prefix over the CTA of one value per thread (kRingThreads threads);
// *cta_total (shared) receives the CTA's total.
__device__ uint64_t block_exclusive(uint64_t v, uint64_t *cta_total) {
    __shared__ uint64_t warp_sums[kRingThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {  // kRingThreads / 32 == 32 warp sums, one per lane
        const uint64_t w = warp_sums[lane];
        uint64_t wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        warp_sums[lane] = wi - w;
        if (lane == 31) *cta_total = wi;
    }
    __syncthreads();
    const uint64_t r = warp_sums[warp] + incl - v;
    __syncthreads();  // warp_sums is reused by the next call
    return r;
}

__device__ __forceinline__ uint32_t record_length(const uint32_t *rings, uint64_t band, uint64_t bands,
                                                  uint32_t reserved) {
    return band < bands ? rings[band * reserved] : 0u;
}

__global__ void __launch_bounds__(kRingThreads)
k_ring_block_sums(const uint32_t *rings, uint64_t bands, uint32_t reserved, uint64_t *block_sums) {
    const uint64_t b0 = (uint64_t)blockIdx.x * kRingChunk + (uint64_t)threadIdx.x * kRingPer;
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < kRingPer; j++) s += record_length(rings, b0 + j, bands, reserved);
    __shared__ uint64_t total;
    block_exclusive(s, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// Exclusive scan of n block sums in place (one CTA); block_sums[n] = the total.
__global__ void __launch_bounds__(kRingThreads) k_ring_scan_blocks(uint64_t *block_sums, uint64_t n) {
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < n; base += kRingThreads) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t v = i < n ? block_sums[i] : 0;
        __shared__ uint64_t total;
        const uint64_t x = block_exclusive(v, &total);
        if (i < n) block_sums[i] = carry + x;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sums[n] = carry;
}

// offsets[band] for every band (and offsets[bands] = total); the in-slot ids of
// every band copied to ids[offsets[band] ..).
__global__ void __launch_bounds__(kRingThreads)
k_ring_gather(const uint32_t *rings, uint64_t bands, uint32_t reserved, const uint64_t *block_base,
              uint64_t *offsets, uint32_t *ids) {
    const uint64_t b0 = (uint64_t)blockIdx.x * kRingChunk + (uint64_t)threadIdx.x * kRingPer;
    uint32_t len[kRingPer];
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < kRingPer; j++) {
        len[j] = record_length(rings, b0 + j, bands, reserved);
        s += len[j];
    }
    __shared__ uint64_t total;
    uint64_t off = block_base[blockIdx.x] + block_exclusive(s, &total);
    uint64_t at[kRingPer];
#pragma unroll
    for (int j = 0; j < kRingPer; j++) {
        at[j] = off;
        if (b0 + j < bands) offsets[b0 + j] = off;
        off += len[j];
    }
    // The warp copies its 32 x kRingPer records one at a time, in band order:
    // lane q moves id q of the record, so each record is one coalesced read of
    // its slots and one contiguous write.
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp_b0 = (uint64_t)blockIdx.x * kRingChunk + (uint64_t)(threadIdx.x & ~31u) * kRingPer;
    for (uint32_t src = 0; src < 32; src++) {
#pragma unroll
        for (int j = 0; j < kRingPer; j++) {
            const uint64_t band = warp_b0 + (uint64_t)src * kRingPer + j;
            const uint32_t n = __shfl_sync(0xffffffffu, min(len[j], reserved - 1), src);
            const uint64_t o = __shfl_sync(0xffffffffu, at[j], src);
            if (band >= bands) continue;  // uniform over the warp
            const uint32_t *rec = rings + band * reserved + 1;
            for (uint32_t q = lane; q < n; q += 32) ids[o + q] = rec[q];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) offsets[bands] = block_base[gridDim.x];
}

// The ids past a band's reserved slots: spill entry (band, slot >= reserved, id)
// is the band's id number slot - 1.
__global__ void k_ring_scatter_spill(const uint4 *spill, uint32_t n, const uint64_t *offsets,
                                     uint32_t *ids) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 s = spill[i];
    const uint64_t band = s.x | ((uint64_t)s.y << 32);
    ids[offsets[band] + s.z - 1] = s.w;
}

}  // namespace

uint64_t ring_scan_blocks(uint64_t bands) { return (bands + kRingChunk - 1) / kRingChunk; }

cudaError_t launch_ring_count(const uint32_t *rings, uint64_t bands, uint32_t reserved,
                              uint64_t *block_sums, cudaStream_t s) {
    const uint64_t nb = ring_scan_blocks(bands);
    if (nb) k_ring_block_sums<<<(unsigned)nb, kRingThreads, 0, s>>>(rings, bands, reserved, block_sums);
    k_ring_scan_blocks<<<1, kRingThreads, 0, s>>>(block_sums, nb);
    return cudaGetLastError();
}

cudaError_t launch_ring_gather(const uint32_t *rings, uint64_t bands, uint32_t reserved,
                               const uint64_t *block_sums, const uint4 *spill, uint32_t n_spill,
                               uint64_t *offsets, uint32_t *ids, cudaStream_t s) {
    const uint64_t nb = ring_scan_blocks(bands);
    if (nb)
        k_ring_gather<<<(unsigned)nb, kRingThreads, 0, s>>>(rings, bands, reserved, block_sums,
                                                          offsets, ids);
    if (n_spill)
        k_ring_scatter_spill<<<(n_spill + 255) / 256, 256, 0, s>>>(spill, n_spill, offsets, ids);
    return cudaGetLastError();
}

}  // namespace tvs
