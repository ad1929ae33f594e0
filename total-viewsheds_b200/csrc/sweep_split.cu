// sweep_split.cu -- the direction-split persistent sweep (layouts 1-9).
//
// The reference kernel (kernel.rs:153-254) walks one band of sight and keeps
// the running maximum of angle = (h - h_pov)/d - d/R; a sample is visible
// when its angle is above the maximum, visible samples add d*tan(1 deg) to
// the band's surface and changes of visibility are ring events.
//
// Mapping.  A CTA sweeps one (sector, tile) item of the work queue
// (queue_sched.cuh).  A warp holds LX columns x 32/LX rows of lanes and each
// lane four points of view (chains), so a warp's 128 chains cover a compact
// patch; the lane sweeps its four forward bands over every step, then its four
// backward bands (the forward surfaces wait in shared memory).  Per step the
// chains of a lane share one table entry and one address (the four samples
// are load immediates apart).
//
// Arithmetic.  Every step first forms the FP32 estimate of the angle from
// the step's tables, a^ = e*y - c (e = RN(h - h_pov), y = RN(1/d),
// c = RN(d/R)), with a per-step window G >= 4 x the estimate's error bound
// (apart from its 2^-22 |a^| part, which the chain's window carries):
//  * FP32 (the comparison form): the estimate is the angle, fma(e, y, -c).
//  * EXACT32 / MIXED64: each chain keeps a window [lo, hi] around its running
//    maximum's estimate and the step j of its maximum.  fma(e, y, -c + G) < lo
//    proves the sample is not visible; fma(e, y, -c - G) > hi proves it is.
//    Only between the two is the comparison re-decided exactly -- in the
//    reference's f32 arithmetic (EXACT32, Markstein division from the table
//    reciprocal) or in FP64 (MIXED64) -- against the exact maximum recomputed
//    from step j.  So every decision is the exact one, and surfaces add the
//    reference's w = RN(d*tan1) in f32 (EXACT32) or RN64(d*0.0174533) in
//    double (MIXED64) in step order: bit for bit the reference f32 sweep and
//    the all-FP64 sweep.
// A warp skips a step when no chain can change state (the vote on the first
// test), and a 32-step segment when the DEM's 16x16 block maxima over the
// warp's patch, moved by the segment's offsets, bound every sample below
// every chain's threshold.
//
// Ring records (kRings): chains keep their previous visibility and record
// count; an event (visibility changed) stores the sample's DEM id in the
// band's next slot, slot 1 is the point of view, slot 0 the count at the end
// (kernel.rs:141-145,220-243).  A chain that was visible at the previous step
// is always evaluated, so its closing event is never skipped.
#include <algorithm>
#include <climits>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include "tvs.h"
#include "tvs_internal.cuh"
#include "queue_sched.cuh"

namespace tvs {
namespace {

constexpr int K = kSplitCols;     // chains per lane
constexpr float kRel = 0x1p-19f;  // the chain window's part relative to |max|

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

// A step's forward DEM offset (cells) as (x, y): |x| < W/2 on every band of
// sight, and |y| <= the line of sight (the shape stage's path check).
__device__ __forceinline__ void step_xy(long long off, long long W, long long &dx, long long &dy) {
    const long long q = off + W / 2;
    dy = q >= 0 ? q / W : -((W - 1 - q) / W);
    dx = off - dy * W;
}

// The quad layout's forward and backward byte offsets of a step from a lane's
// base (copy 0, the group of its first row, its column): rows r0 + y .. +3
// sit in copy (rho + y) mod 4, rho = r0 mod 4 (r0 = the lane's first row).
__device__ __forceinline__ int2 quad_offsets(long long off, long long W, long long rho,
                                             long long copy_bytes) {
    long long dx, dy;
    step_xy(off, W, dx, dy);
    const long long cf = (rho + dy) & 3, cb = (rho - dy) & 3;
    const long long fwd = cf * copy_bytes + (rho + dy - cf) / 4 * W * 16 + dx * 16;
    const long long bwd = cb * copy_bytes + (rho - dy - cb) / 4 * W * 16 - dx * 16;
    return make_int2((int)fwd, (int)bwd);
}

// The per-step window: 2^-20 (d/R + hmax/d) plus a floor, as the shape of
// the estimate's error bound 2^-22 (|a| + d/R + hmax/d) demands (the |a| part
// travels with the chain's maximum).
__device__ __forceinline__ float step_window(float y, float c, float hmax) {
    return __fadd_rn(__fmul_rn(0x1p-20f, __fadd_rn(c, __fmul_rn(hmax, y))), 0x1p-90f);
}

template <int kPrec> struct SplitTypes;
template <> struct SplitTypes<TVS_PRECISION_EXACT32> {
    using S = float;   // surfaces
    using X = float2;  // {d, RN(d/R)}: the exact re-decision
};
template <> struct SplitTypes<TVS_PRECISION_MIXED64> {
    using S = double;
    using X = double2;  // {RN64(d/R), RN64(d*0.0174533)}
};
template <> struct SplitTypes<TVS_PRECISION_FP32> {
    using S = float;
    using X = float2;  // unused
};

// MIXED64 comes in two forms (kLean).  Both keep the step of each chain's
// maximum in registers, two 16-bit steps per register (TVS_MIX_JREG; written
// at every raise, read only by the rare re-decisions).  The default stages
// {RN64(d/R), RN64(d*0.0174533)} per step.  The lean form, for lines of sight
// whose tables would leave fewer than three CTAs per SM, recomputes the
// surface addend from the staged f32 d (one DMUL, the shape stage's own
// operation) and reads RN64(d/R) for the rare exact re-decisions from the FP64
// table in global memory.  Exact f32 holds its running maximum exactly, in
// registers, and evaluates the reference's angle wherever the first test
// passes.
#ifndef TVS_EXACT_INLINE
#define TVS_EXACT_INLINE 1
#endif
// MIXED64 re-decisions read RN64(1/d) from the shape stage's FP64 table
// instead of recomputing it.
#ifndef TVS_MIX_RCP_TABLE
#define TVS_MIX_RCP_TABLE 0
#endif
// MIXED64 keeps the step of each chain's maximum in registers, two 16-bit
// steps per register (band tables of up to 65535 steps; 0 keeps it in shared
// memory instead, 4 B per chain).
#ifndef TVS_MIX_JREG
#define TVS_MIX_JREG 1
#endif

// Shared-memory layout of one CTA.  Every array starts on 16 bytes.
__host__ __device__ constexpr size_t align16(size_t n) { return (n + 15) & ~(size_t)15; }

template <int kPrec, bool kLean = false> struct SplitSmem {
    using S = typename SplitTypes<kPrec>::S;
    using X = typename SplitTypes<kPrec>::X;
    static constexpr bool kExactTab =
        kPrec == TVS_PRECISION_EXACT32 || (kPrec == TVS_PRECISION_MIXED64 && !kLean);
    __host__ __device__ static size_t ctl() { return 0; }
    __host__ __device__ static size_t steps(uint32_t) { return align16(sizeof(QueueCtl)); }
    __host__ __device__ static size_t boff(uint32_t cap) { return steps(cap) + align16((size_t)cap * 16); }
    __host__ __device__ static size_t xtab(uint32_t cap) { return boff(cap) + align16((size_t)cap * 8); }
    __host__ __device__ static size_t seg(uint32_t cap) {
        return xtab(cap) + (kExactTab ? align16((size_t)cap * sizeof(X)) : 0);
    }
    __host__ __device__ static size_t fwd(uint32_t cap) {
        return seg(cap) + align16((size_t)((cap + kSegSteps - 1) / kSegSteps) * sizeof(SegBound));
    }
    __host__ __device__ static size_t jtab(uint32_t cap) {
        return fwd(cap) + (size_t)K * kQueueThreads * sizeof(S);
    }
    __host__ __device__ static size_t total(uint32_t cap) {
        return jtab(cap) + (kPrec == TVS_PRECISION_MIXED64 && !kLean && !TVS_MIX_JREG
                                ? (size_t)K * kQueueThreads * sizeof(int32_t) : 0);
    }
};

// Occupancy target: 4 CTAs of 256 threads per SM (64 registers a thread)
// for the surface sweeps; ring output keeps more state and takes 3.
#ifndef TVS_SPLIT_MIX_BLOCKS
#define TVS_SPLIT_MIX_BLOCKS 4
#endif
#ifndef TVS_SPLIT_BLOCKS32
#define TVS_SPLIT_BLOCKS32 4
#endif
#ifndef TVS_SPLIT_RING_BLOCKS
#define TVS_SPLIT_RING_BLOCKS 3
#endif
#ifndef TVS_SPLIT_RING_BLOCKS32
#define TVS_SPLIT_RING_BLOCKS32 3
#endif
template <int kPrec, bool kRings>
constexpr int split_min_blocks() {
    return (kPrec == TVS_PRECISION_MIXED64 ? (kRings ? TVS_SPLIT_RING_BLOCKS : TVS_SPLIT_MIX_BLOCKS)
                                           : (kRings ? TVS_SPLIT_RING_BLOCKS32 : TVS_SPLIT_BLOCKS32)) *
           8 / kQueueTileY;
}

// Unroll factors of the step loops (FP32 4, exact f32 4, MIXED64 1: the
// fastest on one B200 at 3601^2 within the register budget).
#ifndef TVS_SPLIT_UNROLL32
#define TVS_SPLIT_UNROLL32 4
#endif
#ifndef TVS_SPLIT_UNROLL_EXACT
#define TVS_SPLIT_UNROLL_EXACT 4
#endif
#ifndef TVS_SPLIT_UNROLL_MIX
#define TVS_SPLIT_UNROLL_MIX 1
#endif
#define TVS_PRAGMA(x) _Pragma(#x)
#define TVS_UNROLL(n) TVS_PRAGMA(unroll n)

template <int kPrec, int kLayout, bool kRings, bool kLean>
__global__ void __launch_bounds__(kQueueThreads, (split_min_blocks<kPrec, kRings>()))
k_sweep_split(QueueArgs a) {
    constexpr int LX = split_lx(kLayout), KY = split_ky(kLayout), KX = K / KY, LY = 32 / LX;
    constexpr bool kFp32 = kPrec == TVS_PRECISION_FP32;
    constexpr bool kMix = kPrec == TVS_PRECISION_MIXED64;
    constexpr bool kQuad = kLayout == kQuadLayout;
    using L = SplitSmem<kPrec, kLean>;
    using S = typename L::S;
    using X = typename L::X;
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t cap = a.max_step_cap;
    QueueCtl &ctl = *reinterpret_cast<QueueCtl *>(smem + L::ctl());
    float4 *s_t = reinterpret_cast<float4 *>(smem + L::steps(cap));
    long long *s_boff = reinterpret_cast<long long *>(smem + L::boff(cap));
    int2 *s_q = reinterpret_cast<int2 *>(smem + L::boff(cap));  // quad: {forward, backward}
    X *s_x = reinterpret_cast<X *>(smem + L::xtab(cap));
    SegBound *s_seg = reinterpret_cast<SegBound *>(smem + L::seg(cap));
    S *s_fwd = reinterpret_cast<S *>(smem + L::fwd(cap));
    int32_t *s_j = reinterpret_cast<int32_t *>(smem + L::jtab(cap));  // MIXED64, not lean
    const uint32_t tid = threadIdx.y * kQueueTileX + threadIdx.x;
    const uint32_t lane = threadIdx.x;
    queue_init(ctl, tid);

    while (queue_next(a, ctl, tid)) {
        const QueueDem &D = ctl.dem;
        const uint32_t s = ctl.sector, tile = ctl.tile;
        if (tid < 4) ctl.diag[tid] = 0;
        if (ctl.restage) {
            // ---- stage this DEM's sector tables -----------------------------
            const uint32_t slot = a.first_sector + s;
            const ShapeHeader *h = D.hdr + slot;
            const uint32_t n = h->n_steps;
            const float4 *gs = D.steps + (uint64_t)slot * D.step_cap;
            const int2 *go = D.offs + (uint64_t)slot * D.step_cap;
            const double4 *gd = D.dtab + (uint64_t)slot * D.step_cap;
            const float hmax = kFp32 ? 0.0f : *D.hmax;
            // The quad copies hold a lane's four rows at one column.  The
            // reference's sample ids are linear (kernel.rs:259-292), so a step
            // that moves more than the line of sight sideways wraps a point of
            // view's row; such a sector reads the plain DEM.  Otherwise every
            // point of view's samples stay on its own rows, inside the DEM, and
            // every quad address inside the copies.
            bool plain = !kQuad;
            if constexpr (kQuad) {
                bool wide = false;
                for (uint32_t i = tid; i < n; i += kQueueThreads) {
                    long long dx, dy;
                    step_xy(go[i].x, D.width, dx, dy);
                    wide |= dx > (long long)D.los || dx < -(long long)D.los;
                }
                plain = __syncthreads_or(wide) != 0;
                if (tid == 0) ctl.plain = plain;
            }
            for (uint32_t i = tid; i < n; i += kQueueThreads) {
                const float4 t = gs[i];  // {RN(1/d), d, RN(d/R), RN(d*tan1)}
                if (!plain)
                    s_q[i] = quad_offsets(go[i].x, D.width, (D.row_begin + D.los) & 3u,
                                          (long long)D.quad_copy * 16);
                else
                    s_boff[i] = (long long)go[i].x * (long long)sizeof(float);
                if constexpr (kFp32) {
                    s_t[i] = make_float4(t.x, -t.z, t.w, 0.0f);
                } else {
                    const float g = step_window(t.x, t.z, hmax);
                    const float zhi = __fadd_rn(-t.z, g), zlo = __fsub_rn(-t.z, g);
                    if constexpr (kMix) {
                        s_t[i] = make_float4(t.x, zhi, zlo, t.y);
                        const double4 dt = gd[i];  // {1/d, d/R, d*tan1, d} in double
                        if constexpr (L::kExactTab) s_x[i] = make_double2(dt.y, dt.z);
                    } else {
                        s_t[i] = make_float4(t.x, zhi, zlo, t.w);
                        s_x[i] = make_float2(t.y, t.z);
                    }
                }
            }
            __syncthreads();
            // segment bounds of the fast steps, one warp per segment
            const uint32_t nf = h->n_fast;
            const long long W = D.width;
            for (uint32_t sg = threadIdx.y; sg * kSegSteps < nf; sg += kQueueTileY) {
                const uint32_t i = sg * kSegSteps + lane;
                const bool v = lane < kSegSteps && i < nf;
                long long dxl, dy;
                step_xy(v ? (long long)go[i].x : 0, W, dxl, dy);
                const int dx = (int)dxl;
                int dx0 = v ? dx : INT_MAX, dx1 = v ? dx : INT_MIN;
                int dy0 = v ? (int)dy : INT_MAX, dy1 = v ? (int)dy : INT_MIN;
                float ymax = v ? s_t[i].x : -INFINITY, ymin = v ? s_t[i].x : INFINITY;
                float zmax = v ? s_t[i].y : -INFINITY;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    dx0 = min(dx0, __shfl_xor_sync(0xffffffffu, dx0, o));
                    dx1 = max(dx1, __shfl_xor_sync(0xffffffffu, dx1, o));
                    dy0 = min(dy0, __shfl_xor_sync(0xffffffffu, dy0, o));
                    dy1 = max(dy1, __shfl_xor_sync(0xffffffffu, dy1, o));
                    ymax = fmaxf(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
                    ymin = fminf(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
                    zmax = fmaxf(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
                }
                if (lane == 0) s_seg[sg] = SegBound{dx0, dx1, dy0, dy1, ymax, ymin, zmax, 0.0f};
            }
            if (tid == 0) {
                ctl.sector_status = h->status;
                ctl.n_steps = n;
                ctl.n_fast = nf;
            }
        }
        __syncthreads();  // the staged tables

        if (ctl.sector_status == TVS_OK) {
            const uint32_t n = ctl.n_steps, n_fast = ctl.n_fast;
            const uint32_t bx = tile % D.tiles_x, by = tile / D.tiles_x;
            // chain k: column tx + LX (k % KX), row ty + LY (k / KX)
            const uint32_t lx = lane % LX, ly = lane / LX;
            const uint32_t tx = bx * (KX * LX) + lx;
            const uint32_t ty = D.row_begin + by * (kQueueTileY * LY * KY) + threadIdx.y * LY * KY + ly;
            // rows past the grid are clamped, columns past it read the padding
            // after the elevations; both are discarded (and record no rings)
            auto row_ptr = [&](int r) -> const float * {
                return D.elev + (int64_t)(min(ty + LY * r, D.row_end - 1) + D.los) * D.width + tx + D.los;
            };
            // the quad layout reads the plain DEM only on a few sectors: there
            // the row pointers are recomputed instead of held in registers
            const float *ep[kQuad ? 1 : KY];
#pragma unroll
            for (int r = 0; r < (kQuad ? 1 : KY); r++) ep[r] = row_ptr(r);
            // quad: the lane's base in the row-interleaved copies (rows past the
            // grid are not clamped: the copies hold zero rows for them)
            const char *qbase = nullptr;
            if constexpr (kQuad)
                qbase = reinterpret_cast<const char *>(
                    D.quad + (uint64_t)((ty + D.los - ((D.row_begin + D.los) & 3u)) / 4) * D.width +
                    tx + D.los);
            const int2 *goff = D.offs + (uint64_t)(a.first_sector + s) * D.step_cap;
            const double4 *gdt = D.dtab + (uint64_t)(a.first_sector + s) * D.step_cap;  // MIXED64
            (void)qbase;
            (void)goff;
            (void)gdt;
            float hp32[K];  // kernel.rs:134, the f32 observer elevation
#pragma unroll
            for (int k = 0; k < K; k++)
                hp32[k] = __fadd_rn(__ldg(row_ptr(k / KX) + LX * (k % KX)), D.observer_height);
            // chain k's point-of-view elevation, re-read by the rare exact
            // re-decisions (the address is recomputed rather than kept live)
            auto pov_h = [&](int k) -> float {
                const uint32_t r = min(ty + LY * (k / KX), D.row_end - 1);
                return __ldg(D.elev + (int64_t)(r + D.los) * D.width + tx + LX * (k % KX) + D.los);
            };
            uint32_t active = 0;  // chains on the grid (ring records)
#pragma unroll
            for (int k = 0; k < K; k++)
                if (tx + LX * (k % KX) < D.tvs_width && ty + LY * (k / KX) < D.row_end) active |= 1u << k;
            uint32_t n_swept = 0, n_passed = 0;  // diagnostics (re-decisions count in ctl.diag[3])
            S sb[K];

            // one direction's sweep; PLAIN: a quad-layout sector that reads the
            // plain DEM (a separate instantiation, so that the quad loop is as
            // lean as without it)
            auto pass = [&](auto DIR, auto PLAIN) {
                constexpr int dir = decltype(DIR)::value;
                constexpr bool qplain = decltype(PLAIN)::value;
                auto at = [&](long long b, int k) -> const float * {
                    const float *row = kQuad ? row_ptr(k / KX) : ep[k / KX];
                    return (const float *)((const char *)row + (dir ? -b : b)) + LX * (k % KX);
                };
                // ring records of chain k: kernel id and the DEM id of a sample
                // the four chains' samples at step st
                auto load = [&](uint32_t st, float (&h)[K]) {
                    if constexpr (kQuad && !qplain) {
                        const int2 o = s_q[st];
                        const float4 v = __ldg(reinterpret_cast<const float4 *>(qbase + (dir ? o.y : o.x)));
                        h[0] = v.x;
                        h[1] = v.y;
                        h[2] = v.z;
                        h[3] = v.w;
                    } else {
                        const long long b = s_boff[st];
#pragma unroll
                        for (int k = 0; k < K; k++) h[k] = __ldg(at(b, k));
                    }
                };
                auto load1 = [&](uint32_t st, int k) -> float {
                    if constexpr (kQuad && !qplain) {
                        const int2 o = s_q[st];
                        return __ldg(reinterpret_cast<const float *>(qbase + (dir ? o.y : o.x)) + k);
                    } else {
                        return __ldg(at(s_boff[st], k));
                    }
                };
                // the step's forward offset in bytes in the DEM (ring ids)
                auto orig = [&](uint32_t st) -> long long {
                    if constexpr (kQuad && !qplain)
                        return (long long)__ldg(&goff[st].x) * (long long)sizeof(float);
                    else
                        return s_boff[st];
                };
                // a launch over several sectors keeps each sector's records
                // apart: sector s of the launch owns records s * total_bands ..
                auto kid = [&](int k) -> uint64_t {
                    return (uint64_t)(ty + LY * (k / KX)) * D.tvs_width + tx + LX * (k % KX) +
                           (dir ? a.half_bands : 0) + (uint64_t)s * 2 * a.half_bands;
                };
                auto dem_id = [&](int k, long long b) -> uint32_t {
                    const long long pov = (long long)(ty + LY * (k / KX) + D.los) * D.width +
                                          tx + LX * (k % KX) + D.los;
                    return (uint32_t)(pov + (dir ? -b : b) / (long long)sizeof(float));
                };
                auto ring_put = [&](uint64_t band, uint32_t slot, uint32_t value) {
                    if (slot < a.ring_reserved) {
                        a.rings[band * a.ring_reserved + slot] = value;
                    } else {
                        const uint32_t at_ = atomicAdd(&a.ring_counters[0], 1u);
                        if (at_ < a.spill_cap)
                            a.spill[at_] = make_uint4((uint32_t)band, (uint32_t)(band >> 32), slot, value);
                    }
                };
                uint32_t nr[K];        // ring ids so far (kernel.rs:113 starts at 1)
                uint32_t prev = 0xFu;  // visibility at the previous step (kernel.rs:146)
                if constexpr (kRings) {
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        nr[k] = 1;
                        if (active >> k & 1u) ring_put(kid(k), 1, dem_id(k, 0));  // kernel.rs:145
                    }
                } else {
                    prev = 0;
                }
                auto events = [&](uint32_t vis, uint32_t st) {
                    const uint32_t ev = (vis ^ prev) & active;
                    if (__any_sync(0xffffffffu, ev != 0)) {
                        const long long b = orig(st);
#pragma unroll
                        for (int k = 0; k < K; k++)
                            if (ev >> k & 1u) ring_put(kid(k), ++nr[k], dem_id(k, b));
                    }
                    prev = vis;
                };
                // The largest elevation any lane of this warp samples in a
                // segment: the block maxima over the warp's patch of points of
                // view moved by the segment's offset range (warp-uniform).
                auto segment_max = [&](const SegBound &b) -> float {
                    const int px0 = (int)(bx * (KX * LX) + D.los), px1 = px0 + KX * LX - 1;
                    const int py0 = (int)(D.row_begin + by * (kQueueTileY * LY * KY) +
                                          threadIdx.y * LY * KY + D.los);
                    const int py1 = py0 + LY * KY - 1;
                    const int x0 = dir ? px0 - b.dx1 : px0 + b.dx0, x1 = dir ? px1 - b.dx0 : px1 + b.dx1;
                    const int y0 = dir ? py0 - b.dy1 : py0 + b.dy0, y1 = dir ? py1 - b.dy0 : py1 + b.dy1;
                    const int bx0 = max(x0, 0) / (int)kBlockMax;
                    const int bx1 = min(max(x1, 0) / (int)kBlockMax, (int)D.bmax_w - 1);
                    const int by0 = max(y0, 0) / (int)kBlockMax;
                    const int by1 = min(max(y1, 0) / (int)kBlockMax, (int)D.bmax_h - 1);
                    const int nx = bx1 - bx0 + 1, cells = nx > 0 && by1 >= by0 ? nx * (by1 - by0 + 1) : 0;
                    float m = -INFINITY;
                    for (int q = (int)lane; q < cells; q += 32)
                        m = fmaxf(m, __ldg(D.bmax + (size_t)(by0 + q / nx) * D.bmax_w + bx0 + q % nx));
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                    return m;
                };
                // A segment can be skipped when no chain can change state at
                // any of its steps: every sample h <= B, so e <= RN(B - h_pov)
                // and the first test's value fma(e, y, z) is at most
                // fma(RN(B - h_pov), y_max or y_min, z_max) (RN and fma are
                // monotone).  A chain visible at the previous step must close
                // its ring at the next one, so it is never skipped.
                auto skippable = [&](uint32_t seg, auto &&below) -> bool {
                    const SegBound b = s_seg[seg];
                    const float B = segment_max(b);
                    bool skip = prev == 0;
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        const float E = __fsub_rn(B, hp32[k]);
                        skip &= below(k, __fmaf_rn(E, E >= 0.0f ? b.ymax : b.ymin, b.zmax));
                    }
                    return __all_sync(0xffffffffu, skip);
                };
                S out[K];
                uint32_t i = 0;
                if constexpr (kFp32) {
                    // ---- the reciprocal-table form: the estimate is the angle --
                    float m[K], sf[K];
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        m[k] = kMaxAngle;
                        sf[k] = 0.0f;
                    }
                    auto step = [&](uint32_t st) {
                        const float4 t = s_t[st];  // {y, -c, w, 0}
                        float h[K];
                        load(st, h);
                        uint32_t vis = 0;
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const float ang = __fmaf_rn(__fsub_rn(h[k], hp32[k]), t.x, t.y);
                            const bool v = ang > m[k];
                            if (v) sf[k] = __fadd_rn(sf[k], t.z);
                            m[k] = fmaxf(ang, m[k]);  // NaN yields the other operand
                            vis |= (uint32_t)v << k;
                        }
                        if constexpr (kRings) events(vis, st);
                    };
                    for (uint32_t seg = 0; i < n_fast; seg++) {
                        const uint32_t i1 = min(i + kSegSteps, n_fast);
                        if (skippable(seg, [&](int k, float bound) { return bound <= m[k]; })) {
                            i = i1;
                            continue;
                        }
                        n_swept += i1 - i;
                        TVS_UNROLL(TVS_SPLIT_UNROLL32)
                        for (; i < i1; i++) step(i);
                    }
                    for (; i < n; i++) step(i);  // zero distances: y = inf, the same form
#pragma unroll
                    for (int k = 0; k < K; k++) out[k] = sf[k];
                } else if constexpr (!kMix && TVS_EXACT_INLINE) {
                    // ---- exact f32, the running maximum held exactly ----------
                    // The first test fma(e, y, -c + G) >= m - |m| 2^-19 passes
                    // every step where a chain may change state (|a - (e y - c)|
                    // <= 2^-22 |a| + 2^-23 c); there the reference's angle is
                    // computed for every chain (kernel.rs:175-233).
                    float m[K], lo[K], sf[K];
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        m[k] = kMaxAngle;
                        lo[k] = __fmaf_rn(fabsf(m[k]), -kRel, m[k]);
                        sf[k] = 0.0f;
                    }
                    for (uint32_t seg = 0; i < n_fast; seg++) {
                        const uint32_t i1 = min(i + kSegSteps, n_fast);
                        if (skippable(seg, [&](int k, float bound) { return bound < lo[k]; })) {
                            i = i1;
                            continue;
                        }
                        n_swept += i1 - i;
                        TVS_UNROLL(TVS_SPLIT_UNROLL_EXACT)
                        for (; i < i1; i++) {
                            const float4 t = s_t[i];  // {y, -c + G, -c - G, w}
                            float e[K];
                            load(i, e);
                            bool hit = false;
#pragma unroll
                            for (int k = 0; k < K; k++) {
                                e[k] = __fsub_rn(e[k], hp32[k]);  // kernel.rs:164
                                hit |= __fmaf_rn(e[k], t.x, t.y) >= lo[k];
                            }
                            if (!__any_sync(0xffffffffu, hit || prev != 0)) continue;
                            n_passed++;
                            const float2 x = s_x[i];  // {d, c}
                            uint32_t vis = 0;
#pragma unroll
                            for (int k = 0; k < K; k++) {
                                const float ang = __fsub_rn(div_table32(e[k], t.x, x.x), x.y);
                                const bool v = ang > m[k];
                                if (v) sf[k] = __fadd_rn(sf[k], t.w);
                                m[k] = fmaxf(ang, m[k]);  // f32::max: NaN yields the other
                                lo[k] = __fmaf_rn(fabsf(m[k]), -kRel, m[k]);
                                vis |= (uint32_t)v << k;
                            }
                            if constexpr (kRings) events(vis, i);
                        }
                    }
                    for (; i < n; i++) {  // the zero-distance tail, IEEE division
                        const float2 x = s_x[i];
                        const bool fast = x.x >= 0x1p-20f && x.x <= 0x1p20f;
                        float h[K];
                        load(i, h);
                        uint32_t vis = 0;
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const float e = __fsub_rn(h[k], hp32[k]);
                            const float ang =
                                __fsub_rn(fast ? div_table32(e, s_t[i].x, x.x) : __fdiv_rn(e, x.x), x.y);
                            const bool v = ang > m[k];
                            if (v) sf[k] = __fadd_rn(sf[k], s_t[i].w);
                            m[k] = fmaxf(ang, m[k]);
                            vis |= (uint32_t)v << k;
                        }
                        if constexpr (kRings) events(vis, i);
                    }
#pragma unroll
                    for (int k = 0; k < K; k++) out[k] = sf[k];
                } else {
                    // ---- guard band with exact re-decisions (MIXED64) ----------
                    constexpr bool kJSmem = kMix && !kLean && !TVS_MIX_JREG;
                    constexpr bool kJPack = kMix && TVS_MIX_JREG;
                    float hi[K], lo[K];
                    // step of the running maximum (-1: the initial one)
                    int32_t jreg[kJSmem ? 1 : K] = {};
                    int32_t *sj = s_j + tid;
                    (void)jreg;
                    (void)sj;
                    // packed: two chains' steps per register, 16 bits each
                    // (0xffff: the initial maximum)
                    uint32_t jpk[K / 2] = {};
                    (void)jpk;
                    auto getj = [&](int k) -> int32_t {
                        if constexpr (kJSmem) return sj[k * kQueueThreads];
                        else if constexpr (kJPack) {
                            const uint32_t v = (jpk[k / 2] >> (16 * (k & 1))) & 0xffffu;
                            return v == 0xffffu ? -1 : (int32_t)v;
                        } else return jreg[k];
                    };
                    auto setj = [&](int k, int32_t v) {
                        if constexpr (kJSmem) sj[k * kQueueThreads] = v;
                        else if constexpr (kJPack)
                            jpk[k / 2] = __byte_perm(jpk[k / 2], (uint32_t)v, (k & 1) ? 0x5410 : 0x3254);
                        else jreg[k] = v;
                    };
                    S acc[K];
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        // the initial maximum (-2000, exact) carries the relative part
                        hi[k] = __fmaf_rn(2000.0f, kRel, -2000.0f);
                        lo[k] = __fmaf_rn(2000.0f, -kRel, -2000.0f);
                        setj(k, -1);
                        acc[k] = (S)0;
                    }
                    // the exact angle of chain k at step st, in the precision's arithmetic
                    // MIXED64's per-step FP64 values (fp64_step of the staged d):
                    // the surface addend RN64(d*0.0174533) and RN64(d/R)
                    auto mix_w = [&](uint32_t st) -> double {
                        if constexpr (L::kExactTab) return (double)s_x[st].y;
                        else return __dmul_rn((double)s_t[st].w, 0.0174533);
                    };
                    auto mix_c = [&](uint32_t st) -> double {
                        if constexpr (L::kExactTab) return (double)s_x[st].x;
                        else return __ldg(&gdt[st].y);
                    };
                    auto exact_at = [&](int k, uint32_t st, float h) -> S {
                        if constexpr (kMix) {
                            const double d = (double)s_t[st].w;
                            const double hp64 = __dadd_rn((double)pov_h(k),
                                                          (double)D.observer_height);
                            const double e = __dsub_rn((double)h, hp64);
#if TVS_MIX_RCP_TABLE
                            // the shape stage's RN64(1/d), read instead of recomputed
                            const double y = __ldg(&gdt[st].x);
#else
                            const double y = __drcp_rn(d);
#endif
                            return __dsub_rn(div_table64(e, y, d), mix_c(st));
                        } else {
                            const float e = __fsub_rn(h, hp32[k]);
                            const float2 x = s_x[st];
                            return __fsub_rn(div_table32(e, s_t[st].x, x.x), x.y);
                        }
                    };
                    auto exact_max = [&](int k) -> S {
                        const int32_t j = getj(k);
                        return j < 0 ? (S)kMaxAngle : exact_at(k, (uint32_t)j, load1((uint32_t)j, k));
                    };
                    auto raise = [&](int k, uint32_t st, float fh, float fl, const float4 &t) {
                        hi[k] = __fmaf_rn(fabsf(fh), kRel, fh);
                        lo[k] = __fmaf_rn(fabsf(fl), -kRel, fl);
                        setj(k, (int32_t)st);
                        if constexpr (kMix) acc[k] = __dadd_rn(acc[k], mix_w(st));
                        else acc[k] = __fadd_rn(acc[k], t.w);
                    };
                    for (uint32_t seg = 0; i < n_fast; seg++) {
                        const uint32_t i1 = min(i + kSegSteps, n_fast);
                        if (skippable(seg, [&](int k, float bound) { return bound < lo[k]; })) {
                            i = i1;
                            continue;
                        }
                        n_swept += i1 - i;
                        constexpr int kUnroll = kMix ? TVS_SPLIT_UNROLL_MIX : TVS_SPLIT_UNROLL_EXACT;
#pragma unroll kUnroll
                        for (; i < i1; i++) {
                            const float4 t = s_t[i];  // {y, -c + G, -c - G, w or d}
                            float e[K], fh[K];
                            load(i, e);
                            bool hit = false;
#pragma unroll
                            for (int k = 0; k < K; k++) {
                                e[k] = __fsub_rn(e[k], hp32[k]);  // kernel.rs:164
                                fh[k] = __fmaf_rn(e[k], t.x, t.y);
                                hit |= fh[k] >= lo[k];
                            }
                            if (!__any_sync(0xffffffffu, hit || prev != 0)) continue;
                            n_passed++;
                            uint32_t vis = 0, amb = 0;
                            // the surface addend of this step, read once for the four chains
                            S w;
                            if constexpr (kMix) w = mix_w(i);
                            else w = t.w;
#pragma unroll
                            for (int k = 0; k < K; k++) {
                                const bool maybe = fh[k] >= lo[k];
                                // surely visible: raise the window
                                const float fl = __fmaf_rn(e[k], t.x, t.z);
                                const bool sure = fl > hi[k];
                                if (sure) {
                                    hi[k] = __fmaf_rn(fabsf(fh[k]), kRel, fh[k]);
                                    lo[k] = __fmaf_rn(fabsf(fl), -kRel, fl);
                                    setj(k, (int32_t)i);
                                    if constexpr (kMix) acc[k] = __dadd_rn(acc[k], w);
                                    else acc[k] = __fadd_rn(acc[k], w);
                                }
                                vis |= (uint32_t)sure << k;
                                amb |= (uint32_t)(!sure && maybe) << k;
                            }
                            if (__any_sync(0xffffffffu, amb != 0)) {
                                if (amb) atomicAdd(&ctl.diag[3], (unsigned long long)__popc(amb));
#pragma unroll
                                for (int k = 0; k < K; k++) {
                                    if (!(amb >> k & 1u)) continue;
                                    // kernel.rs:190, decided exactly
                                    if (exact_at(k, i, load1(i, k)) > exact_max(k)) {
                                        raise(k, i, fh[k], __fmaf_rn(e[k], t.x, t.z), t);
                                        vis |= 1u << k;
                                    }
                                }
                            }
                            if constexpr (kRings) events(vis, i);
                        }
                    }
                    // the steps past the table-division domain (the zero
                    // distances): exact arithmetic from the exact maximum
                    S m[K];
#pragma unroll
                    for (int k = 0; k < K; k++) m[k] = exact_max(k);
                    for (; i < n; i++) {
                        float hk[K];
                        load(i, hk);
                        uint32_t vis = 0;
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const float h = hk[k];
                            S ang;
                            if constexpr (kMix) {
                                const double d = (double)s_t[i].w;
                                const double hp64 = __dadd_rn((double)pov_h(k),
                                                              (double)D.observer_height);
                                ang = __dsub_rn(__ddiv_rn(__dsub_rn((double)h, hp64), d), mix_c(i));
                            } else {
                                const float2 x = s_x[i];
                                const bool fast = x.x >= 0x1p-20f && x.x <= 0x1p20f;
                                const float e = __fsub_rn(h, hp32[k]);
                                ang = __fsub_rn(fast ? div_table32(e, s_t[i].x, x.x) : __fdiv_rn(e, x.x), x.y);
                            }
                            const bool v = ang > m[k];
                            if (v) {
                                if constexpr (kMix) acc[k] = __dadd_rn(acc[k], mix_w(i));
                                else acc[k] = __fadd_rn(acc[k], s_t[i].w);
                            }
                            if constexpr (kMix) m[k] = fmax(ang, m[k]);
                            else m[k] = fmaxf(ang, m[k]);  // f32::max: NaN yields the other
                            vis |= (uint32_t)v << k;
                        }
                        if constexpr (kRings) events(vis, i);
                    }
#pragma unroll
                    for (int k = 0; k < K; k++) out[k] = acc[k];
                }
                if constexpr (kRings) {
                    // kernel.rs:237-243: close a ring cut off by the line of
                    // sight, then the count in slot 0
                    const long long b_last = n ? orig(n - 1) : 0;
                    uint32_t most = 0, over = 0;
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        if (!(active >> k & 1u)) continue;
                        if (prev >> k & 1u) ring_put(kid(k), ++nr[k], dem_id(k, b_last));
                        ring_put(kid(k), 0, nr[k]);
                        most = max(most, nr[k]);
                        over += nr[k] >= a.ref_reserved;
                    }
                    most = __reduce_max_sync(0xffffffffu, most);
                    over = __reduce_add_sync(0xffffffffu, over);
                    if (lane == 0) {
                        if (over) atomicAdd(&a.ring_counters[1], over);
                        if (most) atomicMax(&a.ring_counters[2], most);
                    }
                }
#pragma unroll
                for (int k = 0; k < K; k++) {
                    if (dir == 0) s_fwd[k * kQueueThreads + tid] = out[k];
                    else sb[k] = out[k];
                }
            };
            using Fwd = std::integral_constant<int, 0>;
            using Bwd = std::integral_constant<int, 1>;
            using Quad = std::false_type;
            if constexpr (kQuad) {
                if (ctl.plain) {
                    pass(Fwd{}, std::true_type{});
                    pass(Bwd{}, std::true_type{});
                } else {
                    pass(Fwd{}, Quad{});
                    pass(Bwd{}, Quad{});
                }
            } else {
                pass(Fwd{}, Quad{});
                pass(Bwd{}, Quad{});
            }
            if (a.diag || a.rechecks) {
                if (lane == 0) {
                    atomicAdd(&ctl.diag[0], (unsigned long long)n_swept);
                    atomicAdd(&ctl.diag[1], (unsigned long long)n_passed);
                    atomicAdd(&ctl.diag[2], 2ull * n_fast);
                }
            }
            const bool write = queue_wait_prev(a, ctl, D, s, tile, tid);  // every thread
            if (write) {
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const uint32_t col = tx + LX * (k % KX), row = ty + LY * (k / KX);
                    if (col >= D.tvs_width || row >= D.row_end) continue;
                    const uint64_t p = (uint64_t)row * D.tvs_width + col;
                    // forward surface first (kernel.rs:254); in L2: another SM
                    // wrote the previous sector's values
                    if constexpr (kMix) {
                        const double cum = __dadd_rn(
                            __dadd_rn(__ldcg(D.cumulative64 + p), s_fwd[k * kQueueThreads + tid]), sb[k]);
                        __stcg(D.cumulative64 + p, cum);
                        const float c32 = __double2float_rn(cum);
                        __stcg(D.cumulative + p, c32);
                        if (D.total) __stcg(D.total + p, __fadd_rn(__ldcg(D.total + p), c32));
                    } else {
                        const float cum = __fadd_rn(
                            __fadd_rn(__ldcg(D.cumulative + p), s_fwd[k * kQueueThreads + tid]), sb[k]);
                        __stcg(D.cumulative + p, cum);
                        if (D.total) __stcg(D.total + p, __fadd_rn(__ldcg(D.total + p), cum));  // compute.rs:206-214
                    }
                }
            }
            if (tid == 0 && (a.diag || a.rechecks)) {
                if (a.diag) {
                    atomicAdd(&a.diag[0], ctl.diag[0]);
                    atomicAdd(&a.diag[1], ctl.diag[1]);
                    atomicAdd(&a.diag[2], ctl.diag[2]);
                }
                if (a.rechecks && ctl.diag[3]) atomicAdd(a.rechecks, ctl.diag[3]);
            }
        }
        queue_done(a, D, tile, tid);
    }
}

template <int kPrec, int kLayout, bool kRings, bool kLean>
cudaError_t launch_split_t(const QueueArgs &a, cudaStream_t s) {
    const size_t smem = SplitSmem<kPrec, kLean>::total(a.max_step_cap);
    return launch_persistent(
        reinterpret_cast<const void *>(&k_sweep_split<kPrec, kLayout, kRings, kLean>), a, smem, s);
}

template <int kPrec, bool kRings, bool kLean = false>
cudaError_t launch_split_layout(const QueueArgs &a, int layout, cudaStream_t s) {
    switch (layout) {
    case 1: return launch_split_t<kPrec, 1, kRings, kLean>(a, s);
    case 2: return launch_split_t<kPrec, 2, kRings, kLean>(a, s);
    case 3: return launch_split_t<kPrec, 3, kRings, kLean>(a, s);
    case 4: return launch_split_t<kPrec, 4, kRings, kLean>(a, s);
    case 5: return launch_split_t<kPrec, 5, kRings, kLean>(a, s);
    case 6: return launch_split_t<kPrec, 6, kRings, kLean>(a, s);
    case 7: return launch_split_t<kPrec, 7, kRings, kLean>(a, s);
    case 8: return launch_split_t<kPrec, 8, kRings, kLean>(a, s);
    case 9: return launch_split_t<kPrec, 9, kRings, kLean>(a, s);
    default: return cudaErrorInvalidValue;
    }
}

// MIXED64 surfaces run the lean form when it keeps more CTAs per SM (up to
// the register limit) than the default form's tables allow.
cudaError_t mix_lean(uint32_t step_cap, bool *lean) {
    int dev = 0, per_sm = 0, reserved = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (e != cudaSuccess) return e;
    auto ctas = [&](size_t smem) {
        return std::min<size_t>(split_min_blocks<TVS_PRECISION_MIXED64, false>(),
                                (size_t)per_sm / (smem + (size_t)reserved));
    };
    *lean = ctas(SplitSmem<TVS_PRECISION_MIXED64, true>::total(step_cap)) >
            ctas(SplitSmem<TVS_PRECISION_MIXED64>::total(step_cap));
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_persistent(const void *fn, const QueueArgs &a, size_t smem, cudaStream_t s) {
    struct Occ {
        size_t attr = 0, smem = 0;
        int blocks = -1;
    };
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, Occ> occ;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    int blocks_per_sm;
    {
        // contexts on several devices or host threads may launch this kernel
        // concurrently: the attribute only grows, so a launch never finds it
        // below its own shared memory
        std::lock_guard<std::mutex> lock(mu);
        Occ &o = occ[std::make_pair(fn, dev)];
        if (smem > o.attr) {
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            o.attr = smem;
        }
        if (o.blocks < 0 || o.smem != smem) {
            // The resident CTAs at the largest shared-memory carveout, then the
            // smallest carveout that still holds them: the rest of the SM's
            // 256 KB stays L1 cache for the DEM samples (left to itself the
            // driver sizes the carveout for more CTAs than the registers allow).
            int b = 0, per_sm = 0, reserved = 0;
            e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kQueueThreads, smem);
            if (e == cudaSuccess)
                e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
            if (e == cudaSuccess)
                e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
            if (e != cudaSuccess) return e;
            b = b < 1 ? 1 : b;
            if (per_sm > 0) {
                const size_t need = (size_t)b * (smem + (size_t)reserved);
                const int pct = (int)std::min<size_t>(100, (need * 100 + per_sm - 1) / per_sm);
                int b2 = 0;
                e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
                if (e == cudaSuccess)
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, fn, kQueueThreads, smem);
                if (e != cudaSuccess) return e;
                if (b2 < b) {  // the rounding lost a CTA: keep the largest carveout
                    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
                    if (e != cudaSuccess) return e;
                }
            }
            o.blocks = b;
            o.smem = smem;
        }
        blocks_per_sm = o.blocks;
    }
    if (a.done_total > a.done_cap) return cudaErrorInvalidValue;
    e = cudaMemsetAsync(a.queue, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.done, 0, (size_t)a.done_total * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    const uint64_t items = (uint64_t)a.tiles_per_sector * a.n_sectors;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)blocks_per_sm * sms, items);
    QueueArgs args = a;
    void *params[] = {&args};
    e = cudaLaunchKernel(fn, dim3(grid), dim3(kQueueTileX, kQueueTileY), params, smem, s);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

size_t split_smem_bytes(int precision, uint32_t step_cap) {
    switch (precision) {
    case TVS_PRECISION_EXACT32: return SplitSmem<TVS_PRECISION_EXACT32>::total(step_cap);
    case TVS_PRECISION_MIXED64: return SplitSmem<TVS_PRECISION_MIXED64>::total(step_cap);
    case TVS_PRECISION_FP32: return SplitSmem<TVS_PRECISION_FP32>::total(step_cap);
    default: return 0;
    }
}

cudaError_t launch_sweep_split(const QueueArgs &a, int precision, int layout, cudaStream_t s) {
    if (a.n_dems == 0 || a.tiles_per_sector == 0 || a.n_sectors == 0) return cudaSuccess;
    const bool rings = a.rings != nullptr;
    if (rings && (!a.ring_counters || !a.spill || a.ring_reserved < 2))
        return cudaErrorInvalidValue;
    switch (precision) {
    case TVS_PRECISION_EXACT32:
        return rings ? launch_split_layout<TVS_PRECISION_EXACT32, true>(a, layout, s)
                     : launch_split_layout<TVS_PRECISION_EXACT32, false>(a, layout, s);
    case TVS_PRECISION_MIXED64: {
        // 16-bit steps (0xffff marks the initial maximum): at most 65535 steps,
        // a step table of at most 65536 entries (its length rounds up to 4)
        if (TVS_MIX_JREG && a.max_step_cap > 0x10000u) return cudaErrorInvalidValue;
        if (rings) return launch_split_layout<TVS_PRECISION_MIXED64, true>(a, layout, s);
        bool lean = false;
        const cudaError_t e = mix_lean(a.max_step_cap, &lean);
        if (e != cudaSuccess) return e;
        return lean ? launch_split_layout<TVS_PRECISION_MIXED64, false, true>(a, layout, s)
                    : launch_split_layout<TVS_PRECISION_MIXED64, false>(a, layout, s);
    }
    case TVS_PRECISION_FP32:
        return rings ? launch_split_layout<TVS_PRECISION_FP32, true>(a, layout, s)
                     : launch_split_layout<TVS_PRECISION_FP32, false>(a, layout, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace tvs
