// sweep_queue.cu -- persistent band-of-sight sweep over a (sector, tile) work
// queue: the row layouts, and the layout configuration shared with the
// direction-split sweep.
//
// The arithmetic is the reference kernel's (kernel.rs:153-254), as in sweep.cu;
// this file changes how the work is scheduled so that no wave of CTAs runs
// half empty:
//
//  * The grid is exactly the resident capacity of the GPU (occupancy x SMs).
//    Each CTA repeatedly takes the next work item from a global counter.
//  * Items are (sector, tile) pairs in sector-major order, so a CTA mostly
//    stays on one sector and re-stages its step tables in shared memory only
//    when the sector changes.
//  * A tile's sectors must be applied in order (the reference adds sector
//    surfaces to each point's cumulative sum sector by sector, f32).  Each
//    tile has a counter of completed sectors; the item (s, T) waits, after
//    its sweep and before its surface writes, until the counter of T reaches
//    s.  (s-1, T) was dequeued earlier by a CTA that is running, so the wait
//    always ends; it is bounded anyway (spin limit -> TVS_ERR_TIMEOUT in the
//    error word, the item's writes are skipped, the run fails).
//  * Row layouts: a thread sweeps kPx x kPy points of view (columns 32 apart
//    share one address per step through load immediates, rows 8 apart share
//    the table operands); forward and backward bands of a point of view run
//    in the same loop; cum = (cum + forward) + backward keeps the reference's
//    order.  Every step is evaluated.
//  * Direction-split layouts 1-9 live in sweep_split.cu; launch_sweep_queue
//    dispatches to them.
//  * Steps [0, n_fast) use the table division (Markstein, see sweep.cu); the
//    zero-distance tail uses IEEE division.
//
// Precision kPrec: TVS_PRECISION_EXACT32 (reference f32, bit-exact),
// TVS_PRECISION_FP64 (the same control flow in double: angles, maximum and
// surfaces; table division in double from y = RN64(1/d)) or
// TVS_PRECISION_MIXED64 (FP32 estimates, FP64 decisions where the estimate is
// ambiguous and FP64 surfaces: the FP64 results).
#include <algorithm>
#include <climits>
#include <cstdio>
#include <mutex>
#include <cstdlib>
#include <type_traits>

#include "tvs.h"
#include "tvs_internal.cuh"
#include "queue_sched.cuh"

namespace tvs {
namespace {

constexpr int kTileX = kQueueTileX;
constexpr int kTileY = kQueueTileY;
constexpr int kThreads = kQueueThreads;
// the row layouts' tables start 16-byte aligned after the queue control block
__host__ __device__ constexpr size_t row_ctl_bytes() { return (sizeof(QueueCtl) + 15) & ~(size_t)15; }

__device__ __forceinline__ float div_table32(float e, float y, float d) {
    const float q = __fmul_rn(e, y);
    const float r = __fmaf_rn(-d, q, e);
    return __fmaf_rn(r, y, q);
}

__device__ __forceinline__ double div_table64(double e, double y, double d) {
    const double q = __dmul_rn(e, y);
    const double r = __fma_rn(-d, q, e);
    return __fma_rn(r, y, q);
}

// Packed FP32 pairs (sm_100 f32x2): each element is rounded exactly as the
// scalar operation, so a (forward, backward) pair goes through one instruction.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pk(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk(f32x2 v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
// 1.0f when a > b, else 0.0f (false for NaN operands, like the reference's `>`)
__device__ __forceinline__ float gt01(float a, float b) {
    float r;
    asm("set.gt.f32.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// One packed table entry: {y, y}, {-d, -d}, {d/R, d/R}, {d*tan1, d*tan1}.
struct PackedStep {
    f32x2 y, nd, c, w;
};

// Per-point state of one direction.
template <int kPrec> struct Chain;
template <> struct Chain<TVS_PRECISION_EXACT32> {
    float m, s;
    __device__ void init() { m = kMaxAngle; s = 0.0f; }
};
template <> struct Chain<TVS_PRECISION_FP64> {
    double m, s;
    __device__ void init() { m = -2000.0; s = 0.0; }
};
// MIXED64: s is the FP64 surface; m32 is the FP32 estimate of the angle at the
// running maximum, gm the part of the decision window that belongs to it and
// lo = m32 - gm the filter threshold.  The FP64 maximum is the exact angle at
// step j (the last step that raised it; -2000 while j < 0): it is recomputed
// when a comparison needs it and held in m only for the tail steps.
template <> struct Chain<TVS_PRECISION_MIXED64> {
    double m, s;
    float m32, gm, lo;
    int32_t j;
    // the initial maximum carries the |m| 2^-19 part of the window like any other
    __device__ void init() {
        m = -2000.0;
        s = 0.0;
        m32 = -2000.0f;
        gm = 2000.0f * 0x1p-19f;
        lo = __fsub_rn(m32, gm);
        j = -1;
    }
    __device__ void set_max32(float ah, float g) {
        m32 = ah;
        gm = __fmaf_rn(fabsf(ah), 0x1p-19f, g);
        lo = __fsub_rn(m32, gm);
    }
};

template <int kPrec, bool kFast>
__device__ __forceinline__ void step_f32(Chain<kPrec> &c, float h, float hp, const float4 &t,
                                         int slow) {
    const float e = __fsub_rn(h, hp);
    float q;
    if (kFast || !slow) q = div_table32(e, t.x, t.y);
    else q = __fdiv_rn(e, t.y);
    const float a = __fsub_rn(q, t.z);
    if (a > c.m) c.s = __fadd_rn(c.s, t.w);
    c.m = fmaxf(a, c.m);  // f32::max: NaN yields the other operand
}

template <int kPrec, bool kFast>
__device__ __forceinline__ void step_f64(Chain<kPrec> &c, float h, double hp, float d,
                                         const double4 &t, int slow) {
    const double e = __dsub_rn((double)h, hp);
    double q;
    if (kFast || !slow) q = div_table64(e, t.x, (double)d);
    else q = __ddiv_rn(e, (double)d);
    const double a = __dsub_rn(q, t.y);
    if (a > c.m) c.s = __dadd_rn(c.s, t.z);
    c.m = fmax(a, c.m);
}

// MIXED64 carries 6 registers of state per chain; with one or two points of
// view per thread it is held to 64 registers (4 CTAs per SM), with four to 128
// (2 CTAs per SM).
#ifndef TVS_MIX_MIN_BLOCKS
#define TVS_MIX_MIN_BLOCKS 4
#endif
template <int kPrec, int kPx, int kPy>
constexpr int queue_min_blocks() {
    return kPrec != TVS_PRECISION_MIXED64 ? 1
           : kPx * kPy <= 2               ? TVS_MIX_MIN_BLOCKS
           : kPx * kPy == 4               ? 2
                                          : 1;
}

// Row layouts.  kVar: 0 scalar, 1 packed f32x2 (exact f32 only), 2 scalar with
// the next step's elevations loaded while the current step computes.
template <int kPrec, int kPx, int kPy, int kVar>
__global__ void __launch_bounds__(kThreads, (queue_min_blocks<kPrec, kPx, kPy>()))
k_sweep_queue(QueueArgs a) {
    constexpr bool kPacked = kVar == 1;
    constexpr bool kPipe = kVar == 2;
    constexpr bool kMix = kPrec == TVS_PRECISION_MIXED64;
    constexpr bool kF64 = kPrec == TVS_PRECISION_FP64 || kMix;  // FP64 tables and surfaces
    extern __shared__ __align__(16) unsigned char smem[];
    QueueCtl &ctl = *reinterpret_cast<QueueCtl *>(smem);
    float4 *s_steps = reinterpret_cast<float4 *>(smem + row_ctl_bytes());
    // forward DEM-id offset of each step, in bytes (a 64-bit add per base address)
    long long *s_boff = reinterpret_cast<long long *>(s_steps + a.max_step_cap);
    double4 *s_dtab = reinterpret_cast<double4 *>(s_boff + a.max_step_cap);  // FP64 rows only
    PackedStep *s_pk = reinterpret_cast<PackedStep *>(s_boff + a.max_step_cap);  // packed only
    const uint32_t tid = threadIdx.y * kTileX + threadIdx.x;
    queue_init(ctl, tid);

    while (queue_next(a, ctl, tid)) {
        const QueueDem &D = ctl.dem;
        const uint32_t s = ctl.sector, tile = ctl.tile;
        if (ctl.restage) {  // stage this DEM's sector tables
            const uint32_t slot = a.first_sector + s;
            const ShapeHeader *h = D.hdr + slot;
            const uint32_t n = h->n_steps;
            const float4 *gs = D.steps + (uint64_t)slot * D.step_cap;
            const int2 *go = D.offs + (uint64_t)slot * D.step_cap;
            const float hmax = kMix ? *D.hmax : 0.0f;
            for (uint32_t i = tid; i < n; i += kThreads) {
                const float4 t = gs[i];
                s_steps[i] = t;
                if (kMix) {
                    // decision window of the FP32 estimate at this step: at least 4x
                    // the bound 2^-22 (|a| + d/R + hmax/d) on |estimate - FP64 angle|
                    // (the |a| part is carried with the running maximum).  The
                    // filter's offset -d/R + g takes the place of d, which the FP64
                    // table also holds.
                    const float g = __fadd_rn(__fmul_rn(0x1p-20f, __fadd_rn(t.z, __fmul_rn(hmax, t.x))),
                                              0x1p-90f);
                    s_steps[i] = make_float4(t.x, __fadd_rn(-t.z, g), -t.z, g);
                }
                s_boff[i] = (long long)go[i].x * (long long)sizeof(float);
                if (kF64) {
                    s_dtab[i] = D.dtab[(uint64_t)slot * D.step_cap + i];
                } else if (kPacked) {  // only the packed loop reserves these 32 B per step
                    PackedStep p;
                    p.y = pk(t.x, t.x);
                    p.nd = pk(-t.y, -t.y);
                    p.c = pk(t.z, t.z);
                    p.w = pk(t.w, t.w);
                    s_pk[i] = p;
                }
            }
            if (tid == 0) {
                ctl.sector_status = h->status;
                ctl.n_steps = n;
                ctl.n_fast = h->n_fast;
                ctl.hmax = hmax;
            }
        }
        __syncthreads();  // the staged tables
        // The tile's previous sector must be complete before this sector's
        // surfaces are added (bounded wait).  It is awaited after the sweep,
        // by which time it has almost always finished.
        auto wait_prev = [&]() -> bool { return queue_wait_prev(a, ctl, D, s, tile, tid); };
        const bool run = ctl.sector_status == TVS_OK;
        const uint32_t n = ctl.n_steps, n_fast = ctl.n_fast;
        const uint32_t bx = tile % D.tiles_x, by = tile / D.tiles_x;
        const uint32_t tx0 = bx * (kTileX * kPx) + threadIdx.x;
        const uint32_t ty0 = D.row_begin + by * (kTileY * kPy) + threadIdx.y;
        if (run) {
            const float *ep[kPy];
            using HP = typename std::conditional<kF64, double, float>::type;
            HP hp[kPy][kPx];
            float hp32[kPy][kPx];
            Chain<kPrec> cf[kPy][kPx], cb[kPy][kPx];
#pragma unroll
            for (int py = 0; py < kPy; py++) {
                // rows past the grid are clamped, columns past it read padding;
                // both are discarded
                const uint32_t ty = min(ty0 + py * kTileY, D.row_end - 1);
                ep[py] = D.elev + (int64_t)(ty + D.los) * D.width + tx0 + D.los;
#pragma unroll
                for (int px = 0; px < kPx; px++) {
                    const float h0 = __ldg(ep[py] + kTileX * px);
                    if (kF64) hp[py][px] = (HP)__dadd_rn((double)h0, (double)D.observer_height);
                    else hp[py][px] = (HP)__fadd_rn(h0, D.observer_height);  // kernel.rs:134
                    hp32[py][px] = __fadd_rn(h0, D.observer_height);
                    cf[py][px].init();
                    cb[py][px].init();
                }
            }
            // MIXED64 reloads the FP64 observer elevation where it needs it (the
            // rare re-decisions and the tail) instead of holding it
            auto hp_of = [&](int py, int px) -> HP {
                if constexpr (kMix)
                    return (HP)__dadd_rn((double)__ldg(ep[py] + kTileX * px), (double)D.observer_height);
                else
                    return hp[py][px];
            };
            uint32_t i = 0;
            if constexpr (kMix) {
                // FP32 estimate per sample; FP64 only for comparisons inside the
                // window, and for the exact maximum they need (recomputed from
                // the step of the maximum).
                auto exact_angle = [&](int py, int px, int dir, uint32_t k) -> double {
                    const long long bk = s_boff[k];
                    const float *pk_ = (const float *)((const char *)ep[py] + (dir ? -bk : bk));
                    const double ek = __dsub_rn((double)__ldg(pk_ + kTileX * px), hp_of(py, px));
                    const double4 dk = s_dtab[k];
                    return __dsub_rn(div_table64(ek, dk.x, dk.w), dk.y);
                };
                auto max64 = [&](int py, int px, int dir, int32_t j) -> double {
                    return j < 0 ? -2000.0 : exact_angle(py, px, dir, (uint32_t)j);
                };
                // elevations of this step (and, pipelined, of the next one)
                float hc[2][kPy][kPx], hn[2][kPy][kPx];
                auto load_step = [&](float (&h)[2][kPy][kPx], long long b) {
#pragma unroll
                    for (int py = 0; py < kPy; py++)
#pragma unroll
                        for (int px = 0; px < kPx; px++) {
                            h[0][py][px] = __ldg((const float *)((const char *)ep[py] + b) + kTileX * px);
                            h[1][py][px] = __ldg((const float *)((const char *)ep[py] - b) + kTileX * px);
                        }
                };
                if (kPipe && n_fast > 0) load_step(hn, s_boff[0]);
                for (; i < n_fast; i++) {
                    const float4 t = s_steps[i];
                    if constexpr (kPipe) {
#pragma unroll
                        for (int dir = 0; dir < 2; dir++)
#pragma unroll
                            for (int py = 0; py < kPy; py++)
#pragma unroll
                                for (int px = 0; px < kPx; px++) hc[dir][py][px] = hn[dir][py][px];
                        load_step(hn, s_boff[min(i + 1, n_fast - 1)]);
                    } else {
                        load_step(hc, s_boff[i]);
                    }
                    // Filter: a chain can change state at this step only if
                    // estimate + g >= m32 - gm, a superset of the surely-visible
                    // (dd > g) and ambiguous (|dd| <= g) cases below; the window's
                    // slack covers the two extra roundings.  Most steps of most
                    // warps stop here.
                    float es[2][kPy][kPx];
                    bool hit = false;
#pragma unroll
                    for (int py = 0; py < kPy; py++)
#pragma unroll
                        for (int px = 0; px < kPx; px++)
#pragma unroll
                            for (int dir = 0; dir < 2; dir++) {
                                const auto &c = dir ? cb[py][px] : cf[py][px];
                                const float e = __fsub_rn(hc[dir][py][px], hp32[py][px]);
                                es[dir][py][px] = e;
                                hit |= __fmaf_rn(e, t.x, t.y) >= c.lo;
                            }
                    if (!__any_sync(0xffffffffu, hit)) continue;
                    float ahs[2][kPy][kPx], dds[2][kPy][kPx];
#pragma unroll
                    for (int py = 0; py < kPy; py++)
#pragma unroll
                        for (int px = 0; px < kPx; px++)
#pragma unroll
                            for (int dir = 0; dir < 2; dir++) {
                                const auto &c = dir ? cb[py][px] : cf[py][px];
                                ahs[dir][py][px] = __fmaf_rn(es[dir][py][px], t.x, t.z);
                                dds[dir][py][px] = __fsub_rn(ahs[dir][py][px], c.m32);
                            }
                    const double w64 = s_dtab[i].z;
                    bool any_amb = false;
#pragma unroll
                    for (int py = 0; py < kPy; py++)
#pragma unroll
                        for (int px = 0; px < kPx; px++)
#pragma unroll
                            for (int dir = 0; dir < 2; dir++) {
                                auto &c = dir ? cb[py][px] : cf[py][px];
                                const float ah = ahs[dir][py][px], dd = dds[dir][py][px];
                                const bool am = fabsf(dd) <= __fadd_rn(t.w, c.gm);
                                if (!am && dd > 0.0f) {  // surely visible
                                    c.set_max32(ah, t.w);
                                    c.j = (int32_t)i;
                                    c.s = __dadd_rn(c.s, w64);
                                }
                                any_amb |= am;
                            }
                    if (__any_sync(0xffffffffu, any_amb)) {
                        // Re-derive which chains were ambiguous: a chain that was
                        // surely visible at this step has j == i and is skipped;
                        // every other chain still has the state it was tested with.
#pragma unroll
                        for (int py = 0; py < kPy; py++)
#pragma unroll
                            for (int px = 0; px < kPx; px++)
#pragma unroll
                                for (int dir = 0; dir < 2; dir++) {
                                    auto &c = dir ? cb[py][px] : cf[py][px];
                                    if (c.j == (int32_t)i) continue;
                                    const float ah = ahs[dir][py][px], dd = dds[dir][py][px];
                                    if (!(fabsf(dd) <= __fadd_rn(t.w, c.gm))) continue;
                                    if (a.rechecks) atomicAdd(a.rechecks, 1ull);
                                    const double a64 = exact_angle(py, px, dir, i);
                                    if (a64 > max64(py, px, dir, c.j)) {
                                        c.j = (int32_t)i;
                                        c.set_max32(ah, t.w);
                                        c.s = __dadd_rn(c.s, w64);
                                    }
                                }
                    }
                }
                // the exact maximum before the IEEE-division tail
#pragma unroll
                for (int py = 0; py < kPy; py++)
#pragma unroll
                    for (int px = 0; px < kPx; px++)
#pragma unroll
                        for (int dir = 0; dir < 2; dir++) {
                            auto &c = dir ? cb[py][px] : cf[py][px];
                            c.m = max64(py, px, dir, c.j);
                        }
            } else if constexpr (kPipe) {
                float nf[kPy][kPx], nb[kPy][kPx];  // the next step's elevations
                if (n_fast > 0) {
                    const long long b0 = s_boff[0];
#pragma unroll
                    for (int py = 0; py < kPy; py++)
#pragma unroll
                        for (int px = 0; px < kPx; px++) {
                            nf[py][px] = __ldg((const float *)((const char *)ep[py] + b0) + kTileX * px);
                            nb[py][px] = __ldg((const float *)((const char *)ep[py] - b0) + kTileX * px);
                        }
                }
#pragma unroll 2
                for (; i < n_fast; i++) {
                    const float4 t = s_steps[i];
                    double4 dt;
                    if (kF64) dt = s_dtab[i];
                    float hf[kPy][kPx], hb[kPy][kPx];
                    const long long bn = s_boff[min(i + 1, n_fast - 1)];
#pragma unroll
                    for (int py = 0; py < kPy; py++) {
                        const float *pf = (const float *)((const char *)ep[py] + bn);
                        const float *pb = (const float *)((const char *)ep[py] - bn);
#pragma unroll
                        for (int px = 0; px < kPx; px++) {
                            hf[py][px] = nf[py][px];
                            hb[py][px] = nb[py][px];
                            nf[py][px] = __ldg(pf + kTileX * px);
                            nb[py][px] = __ldg(pb + kTileX * px);
                        }
                    }
#pragma unroll
                    for (int py = 0; py < kPy; py++)
#pragma unroll
                        for (int px = 0; px < kPx; px++) {
                            if constexpr (kF64) {
                                step_f64<kPrec, true>(cf[py][px], hf[py][px], hp[py][px], t.y, dt, 0);
                                step_f64<kPrec, true>(cb[py][px], hb[py][px], hp[py][px], t.y, dt, 0);
                            } else {
                                step_f32<kPrec, true>(cf[py][px], hf[py][px], hp[py][px], t, 0);
                                step_f32<kPrec, true>(cb[py][px], hb[py][px], hp[py][px], t, 0);
                            }
                        }
                }
            } else if constexpr (kF64 || !kPacked) {
#pragma unroll 2
                for (; i < n_fast; i++) {
                    const float4 t = s_steps[i];
                    const long long bo = s_boff[i];
                    double4 dt;
                    if (kF64) dt = s_dtab[i];
#pragma unroll
                    for (int py = 0; py < kPy; py++) {
                        const float *pf = (const float *)((const char *)ep[py] + bo);
                        const float *pb = (const float *)((const char *)ep[py] - bo);
#pragma unroll
                        for (int px = 0; px < kPx; px++) {
                            const float hf = __ldg(pf + kTileX * px), hb = __ldg(pb + kTileX * px);
                            if constexpr (kF64) {
                                step_f64<kPrec, true>(cf[py][px], hf, hp[py][px], t.y, dt, 0);
                                step_f64<kPrec, true>(cb[py][px], hb, hp[py][px], t.y, dt, 0);
                            } else {
                                step_f32<kPrec, true>(cf[py][px], hf, hp[py][px], t, 0);
                                step_f32<kPrec, true>(cb[py][px], hb, hp[py][px], t, 0);
                            }
                        }
                    }
                }
            } else {
                // (forward, backward) pairs: e, the table division and the angle
                // packed; visibility as 1.0/0.0 so the surface add is a packed
                // fma (s + 1*w and s + 0*w are exact); maxima stay scalar.
                f32x2 hp2[kPy][kPx], s2[kPy][kPx];
#pragma unroll
                for (int py = 0; py < kPy; py++)
#pragma unroll
                    for (int px = 0; px < kPx; px++) {
                        hp2[py][px] = pk((float)hp[py][px], (float)hp[py][px]);
                        s2[py][px] = pk(0.0f, 0.0f);
                    }
#pragma unroll 2
                for (; i < n_fast; i++) {
                    const PackedStep t = s_pk[i];
                    const long long bo = s_boff[i];
#pragma unroll
                    for (int py = 0; py < kPy; py++) {
                        const float *pf = (const float *)((const char *)ep[py] + bo);
                        const float *pb = (const float *)((const char *)ep[py] - bo);
#pragma unroll
                        for (int px = 0; px < kPx; px++) {
                            const f32x2 e2 = sub2(pk(__ldg(pf + kTileX * px), __ldg(pb + kTileX * px)),
                                                  hp2[py][px]);
                            f32x2 q2 = mul2(e2, t.y);
                            const f32x2 r2 = fma2(t.nd, q2, e2);
                            q2 = fma2(r2, t.y, q2);
                            float af, ab;
                            upk(sub2(q2, t.c), af, ab);
                            auto &F = cf[py][px];
                            auto &B = cb[py][px];
                            s2[py][px] = fma2(pk(gt01(af, F.m), gt01(ab, B.m)), t.w, s2[py][px]);
                            F.m = fmaxf(af, F.m);  // f32::max: NaN yields the other operand
                            B.m = fmaxf(ab, B.m);
                        }
                    }
                }
#pragma unroll
                for (int py = 0; py < kPy; py++)
#pragma unroll
                    for (int px = 0; px < kPx; px++) {
                        float sf_, sb_;
                        upk(s2[py][px], sf_, sb_);
                        cf[py][px].s = sf_;
                        cb[py][px].s = sb_;
                    }
            }
            for (; i < n; i++) {
                const float4 t = s_steps[i];
                const long long bo = s_boff[i];
                double4 dt;
                if (kF64) dt = s_dtab[i];
                const float dist = kMix ? (float)dt.w : t.y;  // MIXED64 keeps d in the FP64 table
                // outside the table-division domain (the zero distances)
                const int slow = !(dist >= 0x1p-20f && dist <= 0x1p20f);
#pragma unroll
                for (int py = 0; py < kPy; py++) {
                    const float *pf = (const float *)((const char *)ep[py] + bo);
                    const float *pb = (const float *)((const char *)ep[py] - bo);
#pragma unroll
                    for (int px = 0; px < kPx; px++) {
                        const float hf = __ldg(pf + kTileX * px);
                        const float hb = __ldg(pb + kTileX * px);
                        if constexpr (kF64) {
                            const double h64 = hp_of(py, px);
                            step_f64<kPrec, false>(cf[py][px], hf, h64, dist, dt, slow);
                            step_f64<kPrec, false>(cb[py][px], hb, h64, dist, dt, slow);
                        } else {
                            step_f32<kPrec, false>(cf[py][px], hf, hp[py][px], t, slow);
                            step_f32<kPrec, false>(cb[py][px], hb, hp[py][px], t, slow);
                        }
                    }
                }
            }
            const bool write = wait_prev();
#pragma unroll
            for (int py = 0; py < kPy; py++) {
                const uint32_t ty = ty0 + py * kTileY;
                if (!write || ty >= D.row_end) continue;
#pragma unroll
                for (int px = 0; px < kPx; px++) {
                    const uint32_t tx = tx0 + kTileX * px;
                    if (tx >= D.tvs_width) continue;
                    const uint64_t p = (uint64_t)ty * D.tvs_width + tx;
                    // surfaces are read and written in L2 (another SM wrote the
                    // previous sector's values)
                    if constexpr (kF64) {
                        const double cum =
                            __dadd_rn(__dadd_rn(__ldcg(D.cumulative64 + p), cf[py][px].s), cb[py][px].s);
                        __stcg(D.cumulative64 + p, cum);
                        const float c32 = __double2float_rn(cum);
                        __stcg(D.cumulative + p, c32);
                        if (D.total) __stcg(D.total + p, __fadd_rn(__ldcg(D.total + p), c32));
                    } else {
                        const float cum =
                            __fadd_rn(__fadd_rn(__ldcg(D.cumulative + p), cf[py][px].s), cb[py][px].s);
                        __stcg(D.cumulative + p, cum);                                  // kernel.rs:254
                        if (D.total) __stcg(D.total + p, __fadd_rn(__ldcg(D.total + p), cum));  // compute.rs:206-214
                    }
                }
            }
        }
        queue_done(a, D, tile, tid);
    }
}

template <int kPrec, int kPx, int kPy, int kVar>
cudaError_t launch_queue_t(const QueueArgs &a, size_t smem, cudaStream_t s) {
    return launch_persistent(reinterpret_cast<const void *>(&k_sweep_queue<kPrec, kPx, kPy, kVar>),
                             a, smem, s);
}

}  // namespace

uint32_t queue_tiles_bound(uint32_t tvs_width, uint32_t rows) {
    // the most tiles any configuration cuts: the row layouts' smallest tile is
    // 32 x 8, but a split layout's tile can be narrower (16 x 64), which on a
    // thin row shard gives more tiles
    auto tiles = [&](uint32_t w, uint32_t h) { return ((tvs_width + w - 1) / w) * ((rows + h - 1) / h); };
    uint32_t n = tiles(kTileX, kTileY);
    for (int l = 1; l <= kSplitLayouts; l++) n = std::max(n, tiles(split_tile_w(l), split_tile_h(l)));
    return n;
}

bool queue_config_valid(const QueueConfig &c) {
    if (c.layout >= 1 && c.layout <= kSplitLayouts)
        return c.px == kSplitCols && c.py == 1 && !c.packed && !c.prefetch;
    if (c.layout != 0) return false;
    const int ok[][2] = {{1, 1}, {2, 1}, {4, 1}, {2, 2}, {8, 1}};
    for (const auto &k : ok)
        if (k[0] == c.px && k[1] == c.py) return true;
    return false;
}

QueueConfig default_queue_config(int precision) {
    static QueueConfig v = [] {
        QueueConfig d{2, 1, 0, 0, 0};
        const char *e = getenv("TVS_SWEEP_SHAPE");
        int x = 0, y = 0;
        if (e && sscanf(e, "%dx%d", &x, &y) == 2) {
            QueueConfig c{x, y, 0, 0, 0};
            if (queue_config_valid(c)) d.px = x, d.py = y;
        }
        const char *p = getenv("TVS_SWEEP_PACKED");
        if (p) d.packed = atoi(p) != 0;
        const char *f = getenv("TVS_SWEEP_PREFETCH");
        if (f) d.prefetch = atoi(f) != 0;
        return d;
    }();
    if (precision == TVS_PRECISION_FP64) return v;
    return default_split_config(precision);
}

QueueConfig default_split_config(int precision) {
    // the fastest split layout per precision on one B200 at 3601^2;
    // TVS_SWEEP_LAYOUT (MIXED64), TVS_SWEEP_LAYOUT32 (exact f32) and
    // TVS_SWEEP_LAYOUT_FP32 override them
    auto env_layout = [](const char *name, int d) {
        const char *l = getenv(name);
        const int v = l ? atoi(l) : d;
        return v >= 1 && v <= kSplitLayouts ? v : d;
    };
    static const int mix = env_layout("TVS_SWEEP_LAYOUT", 1);
    static const int exact = env_layout("TVS_SWEEP_LAYOUT32", kQuadLayout);
    static const int fp32 = env_layout("TVS_SWEEP_LAYOUT_FP32", kQuadLayout);
    const int l = precision == TVS_PRECISION_MIXED64 ? mix
                  : precision == TVS_PRECISION_FP32  ? fp32
                                                     : exact;
    return QueueConfig{kSplitCols, 1, 0, 0, l};
}

void queue_tile(QueueDem *dems, uint32_t n_dems, const QueueConfig &c, uint32_t *tiles_per_sector,
                uint32_t *done_total) {
    uint32_t base = 0;
    for (uint32_t i = 0; i < n_dems; i++) {
        QueueDem &d = dems[i];
        const uint32_t rows = d.row_end - d.row_begin;
        const uint32_t tw = c.layout ? split_tile_w(c.layout) : kTileX * c.px;
        const uint32_t th = c.layout ? split_tile_h(c.layout) : kTileY * c.py;
        d.tiles_x = (d.tvs_width + tw - 1) / tw;
        d.tiles_y = (rows + th - 1) / th;
        d.tile_base = base;
        d.done_base = base;
        base += d.tiles_x * d.tiles_y;
    }
    *tiles_per_sector = base;
    *done_total = base;
}

cudaError_t launch_sweep_queue(const QueueArgs &a, int precision, const QueueConfig &c,
                               cudaStream_t s) {
    if (a.n_dems == 0 || a.tiles_per_sector == 0 || a.n_sectors == 0) return cudaSuccess;
    if (!queue_config_valid(c)) return cudaErrorInvalidValue;
    if (c.layout != 0) {  // direction-split layouts (sweep_split.cu)
        if (precision == TVS_PRECISION_FP64) return cudaErrorInvalidValue;
        return launch_sweep_split(a, precision, c.layout, s);
    }
    const bool mix = precision == TVS_PRECISION_MIXED64;
    const bool f64 = precision == TVS_PRECISION_FP64;
    if (!f64 && !mix && precision != TVS_PRECISION_EXACT32) return cudaErrorInvalidValue;
    if (a.rings) return cudaErrorInvalidValue;  // ring records come from the split layouts
    const bool packed = c.packed && !f64 && !mix;
    const bool pipe = c.prefetch && !packed;
    // ctl + {steps, byte offsets} + FP64 double tables or packed exact-f32 tables
    // (32 B each)
    const bool wide = f64 || mix || packed;
    const size_t smem =
        row_ctl_bytes() + (size_t)a.max_step_cap * (sizeof(float4) + sizeof(long long) + (wide ? 32 : 0));
#define TVS_Q(X, Y)                                                                         \
    if (c.px == X && c.py == Y)                                                             \
        return mix ? (pipe ? launch_queue_t<TVS_PRECISION_MIXED64, X, Y, 2>(a, smem, s)      \
                           : launch_queue_t<TVS_PRECISION_MIXED64, X, Y, 0>(a, smem, s))     \
               : f64 ? (pipe ? launch_queue_t<TVS_PRECISION_FP64, X, Y, 2>(a, smem, s)      \
                             : launch_queue_t<TVS_PRECISION_FP64, X, Y, 0>(a, smem, s))     \
               : packed ? launch_queue_t<TVS_PRECISION_EXACT32, X, Y, 1>(a, smem, s)        \
               : pipe ? launch_queue_t<TVS_PRECISION_EXACT32, X, Y, 2>(a, smem, s)          \
                      : launch_queue_t<TVS_PRECISION_EXACT32, X, Y, 0>(a, smem, s);
    TVS_Q(1, 1) TVS_Q(2, 1) TVS_Q(4, 1) TVS_Q(2, 2) TVS_Q(8, 1)
#undef TVS_Q
    return cudaErrorInvalidValue;
}

}  // namespace tvs
