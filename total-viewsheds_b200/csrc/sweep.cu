// sweep.cu -- band-of-sight sweep kernels.
//
// The reference kernel (crates/shader/src/kernel.rs:71-256) handles one band
// (one point of view, one direction) per invocation: it walks the band's DEM
// ids by the sector's delta table and keeps the running maximum of the
// elevation angle
//     angle = (h - h_pov) / d  -  d / 12742000                 (kernel.rs:175)
// A sample is visible when angle > max (kernel.rs:190); visible samples add
// d * 0.0174533 to the band surface (kernel.rs:216); changes of visibility
// are ring open/close events (kernel.rs:194-229).
//
// The engine kernel here differs in mapping, not in arithmetic:
//  * one thread per point of view runs the forward and the backward band in
//    the same loop (two independent dependency chains), so the reference's
//    "forward bands first, then backward" surface order is kept inside one
//    register: cum = (cum + forward) + backward  (kernel.rs:254);
//  * a CTA is a 32 x 8 tile of points of view; lane = column, so every step
//    reads 32 consecutive elevations (one coalesced 128-byte request);
//  * the step tables are staged in shared memory: the forward DEM-id offset
//    (prefix sum of the deltas, so no serial id chain), 1/d, d, d/R, d*tan1;
//  * a whole run of sectors is one launch: each thread carries its point's
//    cumulative and heatmap-total surfaces across the sectors in registers;
//  * e / d is computed from the table reciprocal y = RN(1/d) as
//    q = RN(e*y), r = fma(-d, q, e), q' = fma(r, y, q).  Markstein's theorem
//    (P. Markstein, IBM J. Res. Dev. 34(1), 1990; also Muller et al.,
//    Handbook of Floating-Point Arithmetic, 2nd ed., section 4.7) gives
//    q' = RN(e/d) when y = RN(1/d), q is within one ulp of e/d and nothing
//    underflows or overflows.  Distances outside [2^-20, 2^20] (the zero
//    distances of unfilled delta-table entries, folded strips) take CUDA's
//    IEEE division instead (a warp-uniform branch: every lane is on the same
//    step).  tvs_selftest_division checks the identity against __fdiv_rn;
//  * delta-table entries the reference never fills (band_of_sight.rs:158
//    fills 2*band_size - band_samples/2 of band_size - 1) have delta 0 and
//    distance 0: the first two give +-inf/NaN angles and can open or close a
//    ring, every later one provably changes nothing (the running maximum
//    already bounds the repeated angle), so the shape stage emits at most two
//    of them and the sweep stops there.
//
// All adds, subtracts and multiplies use the _rn intrinsics so nvcc cannot
// contract them into FMAs; the results are bit-identical to the reference.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>

#include "tvs.h"
#include "tvs_internal.cuh"

namespace tvs {
namespace {

constexpr int kTileX = 32;
constexpr int kTileY = 8;

// RN(e / d) from y = RN(1/d) (Markstein), valid on the table domain.
__device__ __forceinline__ float table_divide(float e, float y, float d) {
    float q = __fmul_rn(e, y);
    float r = __fmaf_rn(-d, q, e);
    return __fmaf_rn(r, y, q);
}

__device__ __forceinline__ void ring_store(const SweepArgs &a, uint64_t kid, uint32_t slot,
                                           uint32_t value) {
    if (slot < a.reserved) {
        a.rings[kid * a.reserved + slot] = value;
    } else {
        uint32_t at = atomicAdd(&a.counters[0], 1u);
        if (at < a.spill_cap)
            a.spill[at] = make_uint4((uint32_t)kid, (uint32_t)(kid >> 32), slot, value);
    }
}

__device__ __forceinline__ void ring_finish(const SweepArgs &a, uint64_t kid, uint32_t n) {
    ring_store(a, kid, 0, n);
    if (n >= (a.ref_reserved ? a.ref_reserved : a.reserved)) atomicAdd(&a.counters[1], 1u);
    atomicMax(&a.counters[2], n);
}

// Loads one sector's step tables into shared memory.  Returns false (for the
// whole CTA) when the sector's shape stage reported an error.
__device__ __forceinline__ bool stage_sector(const SweepArgs &a, uint32_t s, float4 *s_steps,
                                             int2 *s_offs, uint32_t *n_steps) {
    const ShapeHeader *h = a.hdr + s;
    if (h->status != TVS_OK) return false;
    const uint32_t n = h->n_steps;
    const uint32_t tid = threadIdx.y * kTileX + threadIdx.x;
    __syncthreads();  // previous sector's tables are no longer read
    const float4 *gs = a.steps + (uint64_t)s * a.step_cap;
    const int2 *go = a.offs + (uint64_t)s * a.step_cap;
    for (uint32_t i = tid; i < n; i += kTileX * kTileY) {
        s_steps[i] = gs[i];
        s_offs[i] = go[i];
    }
    __syncthreads();
    *n_steps = n;
    return true;
}

template <bool kRings>
__global__ void __launch_bounds__(kTileX * kTileY)
k_sweep_exact32(SweepArgs a) {
    extern __shared__ float4 s_steps[];
    int2 *s_offs = reinterpret_cast<int2 *>(s_steps + a.step_cap);
    const uint32_t tx = blockIdx.x * kTileX + threadIdx.x;
    const uint32_t ty = a.row_begin + blockIdx.y * kTileY + threadIdx.y;
    const bool active = tx < a.tvs_width && ty < a.row_end;
    const uint64_t tvs = (uint64_t)ty * a.tvs_width + tx;
    const int64_t pov = (int64_t)(ty + a.los) * a.width + tx + a.los;
    const float *ep = a.elev + (active ? pov : 0);
    float cum = active ? a.cumulative[tvs] : 0.0f;
    float tot = (active && a.total) ? a.total[tvs] : 0.0f;
    const float hp = __fadd_rn(active ? ep[0] : 0.0f, a.observer_height);  // kernel.rs:134

    for (uint32_t s = 0; s < a.n_sectors; s++) {
        uint32_t n;
        if (!stage_sector(a, s, s_steps, s_offs, &n)) continue;
        if (!active) continue;
        float mf = kMaxAngle, mb = kMaxAngle, sf = 0.0f, sb = 0.0f;
        bool pf = true, pb = true, cf = false, cb = false;
        uint32_t nf = 1, nb = 1;
        int32_t last = 0;
        const uint64_t kf = tvs, kb = tvs + a.half_bands;
        if (kRings) {
            ring_store(a, kf, 1, (uint32_t)pov);  // kernel.rs:145
            ring_store(a, kb, 1, (uint32_t)pov);
        }
#pragma unroll 4
        for (uint32_t i = 0; i < n; i++) {
            const float4 t = s_steps[i];
            const int2 o = s_offs[i];
            const float ef = __fsub_rn(__ldg(ep + o.x), hp);
            const float eb = __fsub_rn(__ldg(ep - o.x), hp);
            float qf, qb;
            if (o.y == 0) {
                qf = table_divide(ef, t.x, t.y);
                qb = table_divide(eb, t.x, t.y);
            } else {
                qf = __fdiv_rn(ef, t.y);
                qb = __fdiv_rn(eb, t.y);
            }
            const float af = __fsub_rn(qf, t.z);
            const float ab = __fsub_rn(qb, t.z);
            const bool vf = af > mf, vb = ab > mb;
            if (vf) sf = __fadd_rn(sf, t.w);
            if (vb) sb = __fadd_rn(sb, t.w);
            if (kRings) {
                if (vf != pf) ring_store(a, kf, ++nf, (uint32_t)(pov + o.x));
                if (vb != pb) ring_store(a, kb, ++nb, (uint32_t)(pov - o.x));
                cf = pf && !vf;
                cb = pb && !vb;
                last = o.x;
            }
            pf = vf;
            pb = vb;
            mf = fmaxf(af, mf);  // f32::max: NaN yields the other operand
            mb = fmaxf(ab, mb);
        }
        if (kRings) {
            if (pf && !cf) ring_store(a, kf, ++nf, (uint32_t)(pov + last));  // kernel.rs:237-240
            if (pb && !cb) ring_store(a, kb, ++nb, (uint32_t)(pov - last));
            ring_finish(a, kf, nf);  // kernel.rs:243
            ring_finish(a, kb, nb);
        }
        cum = __fadd_rn(__fadd_rn(cum, sf), sb);  // kernel.rs:254, forward band first
        tot = __fadd_rn(tot, cum);                // compute.rs:206-214
    }
    if (active) {
        a.cumulative[tvs] = cum;
        if (a.total) a.total[tvs] = tot;
    }
}

// Per-sector launch with the sector's step table in constant memory.  A thread
// sweeps kPx x kPy points of view, both directions: columns tx + 32*px share
// one address per step (the +128*px bytes are load immediates) and rows
// ty + 8*py share the table operands, so each step feeds 2*kPx*kPy independent
// chains.  Steps [0, n_fast) take the table division with no per-step test;
// the rest (the zero-distance tail) test the distance.  Lanes past the
// computable grid sweep a clamped row / an unused column and are discarded;
// the elevation buffer is padded so their loads stay inside the allocation.
__constant__ ShapeHeader c_hdr;
__constant__ float4 c_steps[kConstSteps];
__constant__ int2 c_offs[kConstSteps];

template <int kPx, int kPy>
__global__ void __launch_bounds__(kTileX * kTileY)
k_sweep_exact32_const(SweepArgs a) {
    if (c_hdr.status != TVS_OK) return;
    const uint32_t n = c_hdr.n_steps, n_fast = c_hdr.n_fast;
    const uint32_t tx0 = blockIdx.x * (kTileX * kPx) + threadIdx.x;
    const uint32_t ty0 = a.row_begin + blockIdx.y * (kTileY * kPy) + threadIdx.y;
    const float *ep[kPy];
    float hp[kPy][kPx], mf[kPy][kPx], mb[kPy][kPx], sf[kPy][kPx], sb[kPy][kPx];
#pragma unroll
    for (int py = 0; py < kPy; py++) {
        const uint32_t ty = min(ty0 + py * kTileY, a.row_end - 1);
        ep[py] = a.elev + (int64_t)(ty + a.los) * a.width + tx0 + a.los;
#pragma unroll
        for (int px = 0; px < kPx; px++) {
            hp[py][px] = __fadd_rn(__ldg(ep[py] + kTileX * px), a.observer_height);  // kernel.rs:134
            mf[py][px] = mb[py][px] = kMaxAngle;
            sf[py][px] = sb[py][px] = 0.0f;
        }
    }
    uint32_t i = 0;
#pragma unroll 2
    for (; i < n_fast; i++) {
        const float4 t = c_steps[i];
        const int32_t o = c_offs[i].x;
#pragma unroll
        for (int py = 0; py < kPy; py++) {
            const float *pf = ep[py] + o;
            const float *pb = ep[py] - o;
#pragma unroll
            for (int px = 0; px < kPx; px++) {
                const float af = __fsub_rn(
                    table_divide(__fsub_rn(__ldg(pf + kTileX * px), hp[py][px]), t.x, t.y), t.z);
                const float ab = __fsub_rn(
                    table_divide(__fsub_rn(__ldg(pb + kTileX * px), hp[py][px]), t.x, t.y), t.z);
                if (af > mf[py][px]) sf[py][px] = __fadd_rn(sf[py][px], t.w);
                if (ab > mb[py][px]) sb[py][px] = __fadd_rn(sb[py][px], t.w);
                mf[py][px] = fmaxf(af, mf[py][px]);
                mb[py][px] = fmaxf(ab, mb[py][px]);
            }
        }
    }
    for (; i < n; i++) {
        const float4 t = c_steps[i];
        const int2 o = c_offs[i];
#pragma unroll
        for (int py = 0; py < kPy; py++) {
#pragma unroll
            for (int px = 0; px < kPx; px++) {
                const float ef = __fsub_rn(__ldg(ep[py] + o.x + kTileX * px), hp[py][px]);
                const float eb = __fsub_rn(__ldg(ep[py] - o.x + kTileX * px), hp[py][px]);
                float qf, qb;
                if (o.y == 0) {
                    qf = table_divide(ef, t.x, t.y);
                    qb = table_divide(eb, t.x, t.y);
                } else {
                    qf = __fdiv_rn(ef, t.y);
                    qb = __fdiv_rn(eb, t.y);
                }
                const float af = __fsub_rn(qf, t.z), ab = __fsub_rn(qb, t.z);
                if (af > mf[py][px]) sf[py][px] = __fadd_rn(sf[py][px], t.w);
                if (ab > mb[py][px]) sb[py][px] = __fadd_rn(sb[py][px], t.w);
                mf[py][px] = fmaxf(af, mf[py][px]);
                mb[py][px] = fmaxf(ab, mb[py][px]);
            }
        }
    }
#pragma unroll
    for (int py = 0; py < kPy; py++) {
        const uint32_t ty = ty0 + py * kTileY;
        if (ty >= a.row_end) continue;
#pragma unroll
        for (int px = 0; px < kPx; px++) {
            const uint32_t tx = tx0 + kTileX * px;
            if (tx >= a.tvs_width) continue;
            const uint64_t tvs = (uint64_t)ty * a.tvs_width + tx;
            const float cum = __fadd_rn(__fadd_rn(a.cumulative[tvs], sf[py][px]), sb[py][px]);
            a.cumulative[tvs] = cum;                                   // kernel.rs:254
            if (a.total) a.total[tvs] = __fadd_rn(a.total[tvs], cum);  // compute.rs:206-214
        }
    }
}

// The same control flow with double angles, maximum and surfaces.
template <bool kRings>
__global__ void __launch_bounds__(kTileX * kTileY)
k_sweep_fp64(SweepArgs a) {
    extern __shared__ float4 s_steps[];
    int2 *s_offs = reinterpret_cast<int2 *>(s_steps + a.step_cap);
    const uint32_t tx = blockIdx.x * kTileX + threadIdx.x;
    const uint32_t ty = a.row_begin + blockIdx.y * kTileY + threadIdx.y;
    const bool active = tx < a.tvs_width && ty < a.row_end;
    const uint64_t tvs = (uint64_t)ty * a.tvs_width + tx;
    const int64_t pov = (int64_t)(ty + a.los) * a.width + tx + a.los;
    const float *ep = a.elev + (active ? pov : 0);
    double cum = active ? a.cumulative64[tvs] : 0.0;
    float tot = (active && a.total) ? a.total[tvs] : 0.0f;
    const double hp = __dadd_rn((double)(active ? ep[0] : 0.0f), (double)a.observer_height);

    for (uint32_t s = 0; s < a.n_sectors; s++) {
        uint32_t n;
        if (!stage_sector(a, s, s_steps, s_offs, &n)) continue;
        if (!active) continue;
        double mf = -2000.0, mb = -2000.0, sf = 0.0, sb = 0.0;
        bool pf = true, pb = true, cf = false, cb = false;
        uint32_t nf = 1, nb = 1;
        int32_t last = 0;
        const uint64_t kf = tvs, kb = tvs + a.half_bands;
        if (kRings) {
            ring_store(a, kf, 1, (uint32_t)pov);
            ring_store(a, kb, 1, (uint32_t)pov);
        }
        for (uint32_t i = 0; i < n; i++) {
            const double d = (double)s_steps[i].y;
            const int32_t off = s_offs[i].x;
            const double ef = __dsub_rn((double)__ldg(ep + off), hp);
            const double eb = __dsub_rn((double)__ldg(ep - off), hp);
            const double c = __ddiv_rn(d, 12742000.0);
            const double af = __dsub_rn(__ddiv_rn(ef, d), c);
            const double ab = __dsub_rn(__ddiv_rn(eb, d), c);
            const bool vf = af > mf, vb = ab > mb;
            const double w = __dmul_rn(d, 0.0174533);
            if (vf) sf = __dadd_rn(sf, w);
            if (vb) sb = __dadd_rn(sb, w);
            if (kRings) {
                if (vf != pf) ring_store(a, kf, ++nf, (uint32_t)(pov + off));
                if (vb != pb) ring_store(a, kb, ++nb, (uint32_t)(pov - off));
                cf = pf && !vf;
                cb = pb && !vb;
                last = off;
            }
            pf = vf;
            pb = vb;
            mf = fmax(af, mf);
            mb = fmax(ab, mb);
        }
        if (kRings) {
            if (pf && !cf) ring_store(a, kf, ++nf, (uint32_t)(pov + last));
            if (pb && !cb) ring_store(a, kb, ++nb, (uint32_t)(pov - last));
            ring_finish(a, kf, nf);
            ring_finish(a, kb, nb);
        }
        cum = __dadd_rn(__dadd_rn(cum, sf), sb);
        tot = __fadd_rn(tot, __double2float_rn(cum));
    }
    if (active) {
        a.cumulative64[tvs] = cum;
        a.cumulative[tvs] = __double2float_rn(cum);
        if (a.total) a.total[tvs] = tot;
    }
}

// The plain port of the reference shader: one thread per band, the reference's
// serial delta walk over every entry of the delta table, IEEE divisions.
__device__ __forceinline__ void plain_store(const PlainArgs &a, uint64_t kid, uint32_t slot,
                                            uint32_t value) {
    if (slot < a.reserved) {
        a.rings[kid * a.reserved + slot] = value;
    } else {
        uint32_t at = atomicAdd(&a.counters[0], 1u);
        if (at < a.spill_cap)
            a.spill[at] = make_uint4((uint32_t)kid, (uint32_t)(kid >> 32), slot, value);
    }
}

__global__ void __launch_bounds__(256) k_sweep_plain(PlainArgs a) {
    if (a.hdr->status != TVS_OK) return;
    const uint64_t local_count = (uint64_t)(a.row_end - a.row_begin) * a.tvs_width;
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= 2 * local_count) return;
    const bool backward = j >= local_count;
    const uint64_t local = backward ? j - local_count : j;
    const uint64_t tvs = (uint64_t)a.row_begin * a.tvs_width + local;
    const uint64_t kid = backward ? tvs + a.half_bands : tvs;
    const uint64_t pov_x = tvs % a.tvs_width + a.los;           // kernel.rs:125-131
    const uint64_t pov_y = tvs / a.tvs_width + a.los;
    const int64_t pov = (int64_t)(pov_y * a.width + pov_x);
    const float pov_elevation = __fadd_rn(__ldg(a.elev + pov), a.observer_height);
    float max_angle = kMaxAngle, surface = 0.0f;
    bool cur = true, prev = true, closing = false;
    uint32_t ring_id = 1;
    if (a.rings) plain_store(a, kid, 1, (uint32_t)pov);
    int64_t dem = pov;
    for (uint32_t i = 0; i < a.band_deltas_size; i++) {
        const int32_t delta = __ldg(a.deltas + i);
        dem = backward ? dem - delta : dem + delta;
        const float e = __fsub_rn(__ldg(a.elev + dem), pov_elevation);
        const float d = __ldg(a.dists + i);
        const float angle = __fsub_rn(__fdiv_rn(e, d), __fdiv_rn(d, kEarthRadiusSquared));
        cur = angle > max_angle;
        const bool opening = cur && !prev;
        closing = prev && !cur;
        if (cur) surface = __fadd_rn(surface, __fmul_rn(d, kTanOneRad));
        if (a.rings && (opening || closing)) plain_store(a, kid, ++ring_id, (uint32_t)dem);
        prev = cur;
        max_angle = fmaxf(angle, max_angle);
    }
    if (a.rings) {
        if (cur && !closing) plain_store(a, kid, ++ring_id, (uint32_t)dem);
        plain_store(a, kid, 0, ring_id);
        if (ring_id >= a.reserved) atomicAdd(&a.counters[1], 1u);
        atomicMax(&a.counters[2], ring_id);
    }
    (backward ? a.sb : a.sf)[local] = surface;
}

__global__ void k_combine(float *cum, float *total, const float *sf, const float *sb,
                          uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float c = __fadd_rn(__fadd_rn(cum[i], sf[i]), sb[i]);
    cum[i] = c;
    if (total) total[i] = __fadd_rn(total[i], c);
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ float h_like(uint64_t r) {
    return (float)((int32_t)((r >> 20) & 0xFFFFF) - 0x40000) * 0.03125f;
}

// Random (numerator, distance) pairs: distances log-uniform over the table
// domain [2^-20, 2^20]; numerators either log-uniform over +-[2^-60, 2^60] or
// elevation-like differences (f32 heights minus an observer height).
__global__ void k_selftest_division(uint64_t n, uint64_t seed, unsigned long long *mismatches) {
    unsigned long long local = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r0 = splitmix64(seed ^ (i * 0xD1B54A32D192ED03ull));
        uint64_t r1 = splitmix64(r0);
        uint32_t dexp = 107u + (uint32_t)(r0 % 41u);  // 2^-20 .. 2^20
        float d = __uint_as_float((dexp << 23) | (uint32_t)(r0 >> 41));
        float e;
        if (r1 & 1) {
            uint32_t eexp = 67u + (uint32_t)((r1 >> 1) % 121u);  // 2^-60 .. 2^60
            e = __uint_as_float(((uint32_t)(r1 >> 63) << 31) | (eexp << 23) |
                                (uint32_t)((r1 >> 8) & 0x7FFFFFu));
        } else {
            float h = (float)((int32_t)((r1 >> 8) & 0xFFFFF) - 0x40000) * 0.03125f;
            float hp = __fadd_rn((float)((int32_t)((r1 >> 40) & 0x3FFF) - 0x1000), 1.65f);
            e = __fsub_rn(h, hp);
        }
        float y = __frcp_rn(d);
        float got = table_divide(e, y, d);
        float want = __fdiv_rn(e, d);
        if (__float_as_uint(got) != __float_as_uint(want)) local++;
        // double: numerators with 53 random mantissa bits, the same f32 distances
        uint64_t r2 = splitmix64(r1);
        uint64_t eexp = 1023u - 60u + (r2 % 121u);
        double e64 = __longlong_as_double((long long)(((r2 >> 63) << 63) | (eexp << 52) |
                                                      (splitmix64(r2) >> 12)));
        if (r1 & 2) e64 = __dsub_rn((double)h_like(r2), __dadd_rn((double)h_like(r1), 1.65));
        double d64 = (double)d;
        double q = __dmul_rn(e64, __drcp_rn(d64));
        double r = __fma_rn(-d64, q, e64);
        double got64 = __fma_rn(r, __drcp_rn(d64), q);
        if (__double_as_longlong(got64) != __double_as_longlong(__ddiv_rn(e64, d64))) local++;
    }
    if (local) atomicAdd(mismatches, local);
}

// Eight independent FFMA chains per thread: an FP32 issue-rate probe.
__global__ void __launch_bounds__(256) k_ffma_issue(float *out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = (float)(threadIdx.x + j);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = __fmaf_rn(x[j], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; j++) s = __fadd_rn(s, x[j]);
    if (s == 1234.5f) out[0] = s;  // keeps the chains live
}

// L1 load-throughput probe: every warp reads 32 consecutive floats per load
// (one 128-byte request, the sweep's access) from a 16 KB block-private
// window that stays in L1, eight independent loads in flight per thread.
__global__ void __launch_bounds__(256) k_l1_load(const float *src, float *out, int iters) {
    const float *w = src + (size_t)blockIdx.x * 4096;
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] = 0.0f;
    uint32_t o = threadIdx.x;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] = __fadd_rn(acc[j], __ldg(w + ((o + j * 512u) & 4095u)));
        o = (o + 256u) & 4095u;
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; j++) s = __fadd_rn(s, acc[j]);
    if (s == 1234.5f) out[0] = s;  // keeps the loads live
}

// out[0] = max |x| + |add| (non-negative floats order as their bit patterns).
__global__ void k_max_abs(const float *x, uint64_t n, float add, unsigned int *out) {
    float m = 0.0f;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(__fadd_ru(m, fabsf(add))));
}

__global__ void k_block_max(const float *elev, uint32_t W, uint32_t H, float *bmax) {
    const uint32_t bw = (W + kBlockMax - 1) / kBlockMax, bh = (H + kBlockMax - 1) / kBlockMax;
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bw * bh) return;
    const uint32_t bx = b % bw, by = b / bw;
    float m = -INFINITY;
    for (uint32_t y = by * kBlockMax; y < min(H, (by + 1) * kBlockMax); y++)
        for (uint32_t x = bx * kBlockMax; x < min(W, (bx + 1) * kBlockMax); x++)
            m = fmaxf(m, elev[(uint64_t)y * W + x]);
    bmax[b] = m;
}

// quad[c * per + g * W + x] = rows c + 4g .. c + 4g + 3 of column x (zero
// past the DEM and in the padding after the groups).
__global__ void k_quad_copies(const float *elev, uint32_t W, uint32_t H, uint64_t per,
                              float4 *quad) {
    const uint64_t n = 4 * per, groups = quad_groups(H);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = i / per, r = i - c * per;
        const uint64_t g = r / W, x = r - g * W;
        float v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint64_t row = c + 4 * g + q;
            v[q] = g < groups && row < H ? elev[row * W + x] : 0.0f;
        }
        quad[i] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

__global__ void k_widen(const float *x, double *y, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = (double)x[i];
}

}  // namespace

cudaError_t launch_block_max(const float *elev, uint32_t W, uint32_t H, float *bmax,
                             cudaStream_t s) {
    const uint32_t n = ((W + kBlockMax - 1) / kBlockMax) * ((H + kBlockMax - 1) / kBlockMax);
    if (n == 0) return cudaSuccess;
    k_block_max<<<(n + 255) / 256, 256, 0, s>>>(elev, W, H, bmax);
    return cudaGetLastError();
}

cudaError_t launch_quad_copies(const float *elev, uint32_t W, uint32_t H, float4 *quad,
                               cudaStream_t s) {
    if (W == 0 || H == 0) return cudaSuccess;
    k_quad_copies<<<148 * 8, 256, 0, s>>>(elev, W, H, quad_copy_elems(W, H), quad);
    return cudaGetLastError();
}

cudaError_t launch_widen(const float *x, double *y, uint64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_widen<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, y, n);
    return cudaGetLastError();
}

cudaError_t launch_max_abs(const float *x, uint64_t n, float add, float *out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
    k_max_abs<<<148 * 4, 256, 0, s>>>(x, n, add, reinterpret_cast<unsigned int *>(out));
    return cudaGetLastError();
}

cudaError_t measure_fp32_issue(double *instructions_per_second) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float *out = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(float));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    const int iters = 1 << 14;
    const unsigned blocks = (unsigned)sms * 8u;
    float best = 1e30f;
    for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
        cudaEventRecord(t0);
        k_ffma_issue<<<blocks, 256>>>(out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        if (rep > 0 && ms < best) best = ms;  // the first launch warms up
    }
    if (e == cudaSuccess)
        *instructions_per_second = (double)blocks * 256.0 * iters * 8.0 / (best * 1e-3);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (out) cudaFree(out);
    return e;
}

cudaError_t measure_l1_load(double *bytes_per_second) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned blocks = (unsigned)sms * 4u;
    float *src = nullptr, *out = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&src, (size_t)blocks * 4096 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(src, 0, (size_t)blocks * 4096 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(float));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    const int iters = 1 << 13;
    float best = 1e30f;
    for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
        cudaEventRecord(t0);
        k_l1_load<<<blocks, 256>>>(src, out, iters);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        if (rep > 0 && ms < best) best = ms;  // the first launch warms up
    }
    if (e == cudaSuccess)
        *bytes_per_second = (double)blocks * 256.0 * iters * 8.0 * sizeof(float) / (best * 1e-3);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (src) cudaFree(src);
    if (out) cudaFree(out);
    return e;
}

cudaError_t launch_sweep_engine(const SweepArgs &a, int precision, cudaStream_t s) {
    const uint32_t rows = a.row_end - a.row_begin;
    if (rows == 0 || a.tvs_width == 0 || a.n_sectors == 0) return cudaSuccess;
    dim3 block(kTileX, kTileY);
    dim3 grid((a.tvs_width + kTileX - 1) / kTileX, (rows + kTileY - 1) / kTileY);
    const size_t smem = (size_t)a.step_cap * (sizeof(float4) + sizeof(int2));
    const bool rings = a.rings != nullptr;
    void (*fn)(SweepArgs);
    // MIXED64 decides every comparison as the FP64 sweep does, so the FP64
    // kernel produces its ring records and surfaces
    if (precision == TVS_PRECISION_FP64 || precision == TVS_PRECISION_MIXED64)
        fn = rings ? k_sweep_fp64<true> : k_sweep_fp64<false>;
    else if (precision == TVS_PRECISION_EXACT32)
        fn = rings ? k_sweep_exact32<true> : k_sweep_exact32<false>;
    else
        return cudaErrorInvalidValue;
    cudaError_t e = grow_smem_attribute(reinterpret_cast<const void *>(fn), smem);
    if (e != cudaSuccess) return e;
    fn<<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t grow_smem_attribute(const void *fn, size_t smem) {
    // The attribute belongs to (kernel, device).  Host threads and contexts on
    // several devices launch the same kernels with different line-of-sight
    // lengths, so the attribute is only ever raised: a launch never finds it
    // below the shared memory it asks for, whatever another thread set since.
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> attr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = attr[std::make_pair(fn, dev)];
    if (smem <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) cur = smem;
    return e;
}

// Points of view per thread of the constant-table sweep: columns x rows.
// TVS_SWEEP_SHAPE ("4x1", "2x2", "2x1", "1x2", "1x1", "8x1") overrides the default
// for tuning runs.
struct PovShape { int px, py; };

PovShape const_shape() {
    static PovShape v = [] {
        const char *e = getenv("TVS_SWEEP_SHAPE");
        PovShape d{4, 1};
        if (!e) return d;
        int x = 0, y = 0;
        if (sscanf(e, "%dx%d", &x, &y) != 2) return d;
        const PovShape ok[] = {{1, 1}, {2, 1}, {1, 2}, {2, 2}, {4, 1}, {8, 1}, {4, 2}};
        for (const PovShape &k : ok)
            if (k.px == x && k.py == y) return k;
        return d;
    }();
    return v;
}

cudaError_t launch_sweep_const(const SweepArgs &a, int precision, uint32_t n_steps,
                               cudaStream_t s) {
    if (precision != TVS_PRECISION_EXACT32 || a.rings || a.n_sectors != 1 || n_steps > kConstSteps)
        return cudaErrorInvalidValue;
    const uint32_t rows = a.row_end - a.row_begin;
    if (rows == 0 || a.tvs_width == 0) return cudaSuccess;
    cudaError_t e = cudaMemcpyToSymbolAsync(c_hdr, a.hdr, sizeof(ShapeHeader), 0,
                                            cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && n_steps)
        e = cudaMemcpyToSymbolAsync(c_steps, a.steps, n_steps * sizeof(float4), 0,
                                    cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && n_steps)
        e = cudaMemcpyToSymbolAsync(c_offs, a.offs, n_steps * sizeof(int2), 0,
                                    cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    const PovShape sh = const_shape();
    dim3 block(kTileX, kTileY);
    dim3 grid((a.tvs_width + kTileX * sh.px - 1) / (kTileX * sh.px),
              (rows + kTileY * sh.py - 1) / (kTileY * sh.py));
#define TVS_CONST_CASE(X, Y) \
    if (sh.px == X && sh.py == Y) k_sweep_exact32_const<X, Y><<<grid, block, 0, s>>>(a); else
    TVS_CONST_CASE(1, 1) TVS_CONST_CASE(2, 1) TVS_CONST_CASE(1, 2) TVS_CONST_CASE(2, 2)
    TVS_CONST_CASE(8, 1) TVS_CONST_CASE(4, 2)
    k_sweep_exact32_const<4, 1><<<grid, block, 0, s>>>(a);
#undef TVS_CONST_CASE
    return cudaGetLastError();
}

cudaError_t launch_sweep_plain(const PlainArgs &a, cudaStream_t s) {
    const uint64_t n = 2ull * (a.row_end - a.row_begin) * a.tvs_width;
    if (n == 0) return cudaSuccess;
    k_sweep_plain<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_combine(float *cum, float *total, const float *sf, const float *sb,
                           uint64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_combine<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cum, total, sf, sb, n);
    return cudaGetLastError();
}

cudaError_t launch_selftest_division(uint64_t n, uint64_t seed, unsigned long long *mismatches,
                                     cudaStream_t s) {
    k_selftest_division<<<148 * 8, 256, 0, s>>>(n, seed, mismatches);
    return cudaGetLastError();
}

}  // namespace tvs
