// shape.cu -- per-sector band-of-sight shape stage (one CTA per sector).
//
// Reference: Axes::compute (axes.rs:103-130) sorts all W*H points twice per
// sector (FP64 projection, f32 cast, stable radix sort) and
// DEM::compile_band_data (band_of_sight.rs:61-174) then reads only a window of
// band_samples ranks around the DEM centre from the sector order, re-ordered
// by sight rank.  This kernel produces exactly that window without a full sort:
//
//  1. Along one DEM row the sector projection x*sin - y*cos is monotone in x,
//     and so are its f32 cast and radix key.  The number of points with key < K
//     is therefore a sum of per-row binary searches (H * log2(W) evaluations
//     instead of W*H).
//  2. A binary search over the 32-bit key space finds the keys K_lo, K_hi of
//     the first and last window ranks, and count(key < K_lo).
//  3. The points with K_lo <= key <= K_hi (the window plus key ties) are
//     gathered into shared memory and sorted by (key, id): radsort is stable,
//     so this is exactly the reference's sector order on those ranks.
//  4. The window is sorted by (sight key, id), which orders it by
//     sight_ordered_map rank (band_of_sight.rs:135-145), and the delta and
//     distance tables are derived from the strip (band_of_sight.rs:149-170).
//  5. The sweep's per-step tables (forward offsets, 1/d, d/R, d*tan1) follow.
//
// Every projection is rounded op by op (__dmul_rn/__dsub_rn), with host glibc
// sin/cos, so keys are bitwise those of the reference.
#include "tvs.h"
#include "tvs_internal.cuh"

namespace tvs {
namespace {

// axes.rs:160-171: y runs 0, -1, ..., -(H-1) (row 0 gives +0.0).
__device__ __forceinline__ double row_term(uint32_t row, double c) {
    return __dmul_rn((double)(-(int64_t)row), c);
}

__device__ __forceinline__ float projection32(uint32_t x, double right, double s) {
    return __double2float_rn(__dsub_rn(__dmul_rn((double)x, s), right));
}

__device__ __forceinline__ uint32_t key_at(uint32_t x, double right, double s) {
    return f32_radix_key(projection32(x, right, s));
}

// Number of x in [x0, x0 + S) whose key is < K.  Keys are non-decreasing in x
// when s >= 0 and non-increasing when s < 0.
__device__ uint32_t row_count_less(uint64_t K, double right, double s, uint32_t x0, uint32_t S) {
    uint32_t lo = 0, hi = S;
    if (!(s < 0.0)) {
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if ((uint64_t)key_at(x0 + mid, right, s) < K) lo = mid + 1; else hi = mid;
        }
        return lo;
    }
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if ((uint64_t)key_at(x0 + mid, right, s) < K) hi = mid; else lo = mid + 1;
    }
    return S - lo;
}

template <typename T>
__device__ T block_sum(T v, T *scratch) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T r = 0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; w++) r += scratch[w];
    return r;
}

// Sum over the rows of the window of count(key < K), two thresholds at once.
__device__ void count_less2(uint64_t K0, uint64_t K1, double c, double s, uint32_t x0,
                            uint32_t y0, uint32_t S, uint64_t *out0, uint64_t *out1,
                            unsigned long long *scratch) {
    unsigned long long a = 0, b = 0;
    for (uint32_t r = threadIdx.x; r < S; r += blockDim.x) {
        double right = row_term(y0 + r, c);
        a += row_count_less(K0, right, s, x0, S);
        b += row_count_less(K1, right, s, x0, S);
    }
    *out0 = block_sum(a, scratch);
    *out1 = block_sum(b, scratch + 32);
}

__device__ void bitonic_sort(unsigned long long *v, uint32_t n_pow2) {
    for (uint32_t k = 2; k <= n_pow2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < n_pow2; i += blockDim.x) {
                uint32_t ixj = i ^ j;
                if (ixj > i) {
                    unsigned long long a = v[i], b = v[ixj];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) { v[i] = b; v[ixj] = a; }
                }
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ uint32_t next_pow2(uint32_t n) {
    uint32_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Inclusive prefix sum of n int64 values in place (one CTA).
__device__ void block_inclusive_scan(long long *v, uint32_t n, long long *scratch) {
    const uint32_t T = blockDim.x;
    const uint32_t per = (n + T - 1) / T;
    const uint32_t b = threadIdx.x * per;
    const uint32_t e = min(n, b + per);
    long long local = 0;
    for (uint32_t i = b; i < e; i++) local += v[i];
    // exclusive scan of the per-thread sums through shared memory
    __syncthreads();
    scratch[threadIdx.x] = local;
    __syncthreads();
    for (uint32_t off = 1; off < T; off <<= 1) {
        long long add = threadIdx.x >= off ? scratch[threadIdx.x - off] : 0;
        __syncthreads();
        scratch[threadIdx.x] += add;
        __syncthreads();
    }
    long long run = scratch[threadIdx.x] - local;
    for (uint32_t i = b; i < e; i++) { run += v[i]; v[i] = run; }
    __syncthreads();
}

struct ShapeSmem {
    unsigned long long red[64];
    long long scan[kShapeThreads];
    uint32_t n_cand;
    int32_t status;
};

}  // namespace

// Steps 5-7: the sweep's step tables from the prefix-summed forward offsets
// soff[0, n_filled) and distances sdist[0, n_filled) in shared memory, the
// path-bounds status and the header.  Steps past n_filled repeat the last
// offset with d = 0.
__device__ void finish_shape(const ShapeArgs &a, uint32_t sector, uint32_t n_filled,
                             uint32_t n_steps, uint32_t n_cand, const long long *soff,
                             const float *sdist, ShapeSmem &sm) {
    ShapeHeader *hdr = a.hdr + sector;
    long long mn = 0, mx = 0;
    uint32_t first_slow = n_steps;
    float4 *gsteps = a.steps + (uint64_t)sector * a.step_cap;
    int2 *goffs = a.offs + (uint64_t)sector * a.step_cap;
    for (uint32_t i = threadIdx.x; i < n_steps; i += blockDim.x) {
        long long off = i < n_filled ? soff[i] : (n_filled ? soff[n_filled - 1] : 0);
        float d = i < n_filled ? sdist[i] : 0.0f;
        float4 st;
        st.x = __frcp_rn(d);
        st.y = d;
        st.z = __fdiv_rn(d, kEarthRadiusSquared);
        st.w = __fmul_rn(d, kTanOneRad);
        int flags = (d >= 0x1p-20f && d <= 0x1p20f) ? 0 : kStepSlowDivide;
        gsteps[i] = st;
        goffs[i] = make_int2((int32_t)off, flags);
        // FP64 sweep tables: the same distance in double (kernel.rs:175,216)
        a.dtab[(uint64_t)sector * a.step_cap + i] = fp64_step(d);
        mn = min(mn, off);
        mx = max(mx, off);
        if (flags) first_slow = min(first_slow, i);
    }
    __syncthreads();
    sm.scan[threadIdx.x] = first_slow;
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm.scan[threadIdx.x] = min(sm.scan[threadIdx.x], sm.scan[threadIdx.x + o]);
        __syncthreads();
    }
    const uint32_t n_fast = (uint32_t)sm.scan[0];
    __syncthreads();
    // block min / max through the scan scratch
    sm.scan[threadIdx.x] = mn;
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm.scan[threadIdx.x] = min(sm.scan[threadIdx.x], sm.scan[threadIdx.x + o]);
        __syncthreads();
    }
    const long long min_off = sm.scan[0];
    __syncthreads();
    sm.scan[threadIdx.x] = mx;
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm.scan[threadIdx.x] = max(sm.scan[threadIdx.x], sm.scan[threadIdx.x + o]);
        __syncthreads();
    }
    const long long max_off = sm.scan[0];
    if (threadIdx.x == 0) {
        // kernel.rs:157-164: every band of every point of view stays on the DEM.
        const long long size = (long long)a.size;
        bool ok = a.pov_min + min_off >= 0 && a.pov_max + max_off < size &&
                  a.pov_min - max_off >= 0 && a.pov_max - min_off < size &&
                  min_off >= INT32_MIN && max_off <= INT32_MAX;
        hdr->status = ok ? TVS_OK : TVS_ERR_PATH_OUT_OF_DEM;
        hdr->n_filled = n_filled;
        hdr->n_steps = n_steps;
        hdr->n_candidates = n_cand;
        hdr->min_off = min_off;
        hdr->max_off = max_off;
        hdr->n_fast = n_fast;
    }}

// One sector of one DEM (the whole CTA).
__device__ __forceinline__ void shape_sector(const ShapeArgs &a, const uint32_t sector,
                                             const uint64_t rank_lo, const uint64_t rank_count,
                                             const int axes_mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ShapeSmem &sm = *reinterpret_cast<ShapeSmem *>(smem_raw);
    unsigned long long *cand = reinterpret_cast<unsigned long long *>(smem_raw + sizeof(ShapeSmem));
    unsigned long long *win = cand + kCandidateCap;

    const SectorTrig tr = a.trig[sector];
    const uint32_t W = a.width;
    const uint32_t S = a.win, X0 = a.x0, Y0 = a.y0;
    const uint64_t rank_hi = rank_lo + rank_count - 1;

    // 1-2. Keys of ranks rank_lo and rank_hi in the sector order.
    uint64_t lo0 = 0, hi0 = 0xFFFFFFFFull, lo1 = 0, hi1 = 0xFFFFFFFFull;
    for (int it = 0; it < 33 && (lo0 < hi0 || lo1 < hi1); it++) {
        uint64_t mid0 = lo0 + ((hi0 - lo0) >> 1);
        uint64_t mid1 = lo1 + ((hi1 - lo1) >> 1);
        uint64_t c0, c1;
        count_less2(mid0 + 1, mid1 + 1, tr.sector_cos, tr.sector_sin, X0, Y0, S, &c0, &c1, sm.red);
        if (lo0 < hi0) { if (c0 > rank_lo) hi0 = mid0; else lo0 = mid0 + 1; }
        if (lo1 < hi1) { if (c1 > rank_hi) hi1 = mid1; else lo1 = mid1 + 1; }
    }
    const uint64_t K_lo = lo0, K_hi = lo1;
    uint64_t less_lo, le_hi;
    count_less2(K_lo, K_hi + 1, tr.sector_cos, tr.sector_sin, X0, Y0, S, &less_lo, &le_hi, sm.red);

    // 3. Gather the candidates (every point with K_lo <= key <= K_hi).
    if (threadIdx.x == 0) { sm.n_cand = 0; sm.status = TVS_OK; }
    __syncthreads();
    const bool inc = !(tr.sector_sin < 0.0);
    for (uint32_t r = threadIdx.x; r < S; r += blockDim.x) {
        const uint32_t row = Y0 + r;
        double right = row_term(row, tr.sector_cos);
        uint32_t b = row_count_less(K_lo, right, tr.sector_sin, X0, S);
        uint32_t e = row_count_less(K_hi + 1, right, tr.sector_sin, X0, S);
        if (e <= b) continue;
        uint32_t x0 = X0 + (inc ? b : S - e);
        uint32_t n = e - b;
        uint32_t at = atomicAdd(&sm.n_cand, n);
        for (uint32_t k = 0; k < n; k++) {
            if (at + k >= kCandidateCap) break;
            uint32_t x = x0 + k;
            uint32_t id = row * W + x;
            cand[at + k] = ((unsigned long long)key_at(x, right, tr.sector_sin) << 32) | id;
        }
    }
    __syncthreads();
    const uint32_t n_cand = sm.n_cand;
    ShapeHeader *hdr = a.hdr + sector;
    if (n_cand > kCandidateCap || less_lo > rank_lo ||
        (rank_lo - less_lo) + rank_count > n_cand) {
        if (threadIdx.x == 0) {
            hdr->status = n_cand > kCandidateCap ? TVS_ERR_CAPACITY : TVS_ERR_SHAPE;
            hdr->n_candidates = n_cand;
            hdr->n_filled = hdr->n_steps = 0;
        }
        return;
    }
    const uint32_t pc = next_pow2(n_cand);
    for (uint32_t i = n_cand + threadIdx.x; i < pc; i += blockDim.x) cand[i] = ~0ull;
    __syncthreads();
    bitonic_sort(cand, pc);
    const uint32_t start = (uint32_t)(rank_lo - less_lo);

    if (axes_mode) {
        for (uint32_t j = threadIdx.x; j < rank_count; j += blockDim.x)
            a.sector_ids_out[j] = (uint32_t)cand[start + j];
        if (threadIdx.x == 0) { hdr->status = TVS_OK; hdr->n_candidates = n_cand; }
        return;
    }

    // 4. Order the window by sight rank == (sight key, id).
    const uint32_t bs = a.band_samples;
    for (uint32_t j = threadIdx.x; j < bs; j += blockDim.x) {
        uint32_t id = (uint32_t)cand[start + j];
        uint32_t row = id / W, x = id - row * W;
        float d = projection32(x, row_term(row, tr.sight_cos), tr.sight_sin);
        win[j] = ((unsigned long long)f32_radix_key(d) << 32) | id;
    }
    const uint32_t pw = next_pow2(bs);
    for (uint32_t i = bs + threadIdx.x; i < pw; i += blockDim.x) win[i] = ~0ull;
    __syncthreads();
    bitonic_sort(win, pw);

    // band_of_sight.rs:149-170 (the geometry checks on the host guarantee
    // middle < end <= band_samples - 1 and filled <= band_deltas_size).
    const uint32_t middle = bs / 2;
    const uint32_t n_filled = 2 * a.band_size - middle;
    const uint32_t bds = a.band_deltas_size;
    const uint32_t n_steps = n_filled + min(bds - n_filled, 2u);
    long long *soff = reinterpret_cast<long long *>(cand);           // reuse candidates
    float *sdist = reinterpret_cast<float *>(soff + bds + 2);
    // band_of_sight.rs:99: the middle point of the (window's) row-major order
    const uint64_t pov_local = (uint64_t)S * S / 2;
    const uint32_t pov_id = (uint32_t)((Y0 + pov_local / S) * (uint64_t)W + X0 + pov_local % S);
    const float pov_distance =
        projection32(pov_id % W, row_term(pov_id / W, tr.sight_cos), tr.sight_sin);
    int32_t *gdel = a.deltas + (uint64_t)sector * bds;
    float *gdist = a.dists + (uint64_t)sector * bds;
    for (uint32_t i = threadIdx.x; i < bds; i += blockDim.x) {
        int32_t delta = 0;
        float dist = 0.0f;
        if (i < n_filled) {
            uint32_t cur = (uint32_t)win[middle + i];
            uint32_t nxt = (uint32_t)win[middle + i + 1];
            delta = (int32_t)cur - (int32_t)nxt;
            uint32_t row = nxt / W, x = nxt - row * W;
            float nd = projection32(x, row_term(row, tr.sight_cos), tr.sight_sin);
            dist = fabsf(__fsub_rn(pov_distance, nd));
        }
        gdel[i] = delta;
        gdist[i] = dist;
        if (i < n_filled) { soff[i] = delta; sdist[i] = dist; }
    }
    __syncthreads();
    block_inclusive_scan(soff, n_filled, sm.scan);

    finish_shape(a, sector, n_filled, n_steps, n_cand, soff, sdist, sm);
}

__global__ void __launch_bounds__(kShapeThreads, 1)
k_shape(ShapeArgs a, uint64_t rank_lo, uint64_t rank_count, int axes_mode) {
    shape_sector(a, blockIdx.x, rank_lo, rank_count, axes_mode);
}

// Many DEMs at once: CTA b handles sector b % n_sectors of DEM b / n_sectors.
__global__ void __launch_bounds__(kShapeThreads, 1)
k_shape_batch(const ShapeArgs *args, uint32_t n_sectors) {
    const ShapeArgs a = args[blockIdx.x / n_sectors];
    const uint64_t m = (uint64_t)a.win * a.win;
    shape_sector(a, blockIdx.x % n_sectors, m / 2 - a.band_samples / 2, a.band_samples, 0);
}

// A band shape given as tables instead of computed: the reference's shape
// cache (cache.rs:50-60, read at compute.rs:132-140) holds the deltas and
// distances of compile_band_data.  Sector b of the launch takes them from
// tab_deltas/tab_dists + b * band_deltas_size when installed[b] != 0 and
// overwrites the computed shape with them; its step tables follow as for a
// computed shape.  The filled length is one past the last entry with a
// nonzero delta or a distance other than +0 (the host has checked it against
// the step-table capacity).
__global__ void __launch_bounds__(kShapeThreads, 1)
k_shape_tables(ShapeArgs a, const int32_t *tab_deltas, const float *tab_dists,
               const unsigned char *installed) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ShapeSmem &sm = *reinterpret_cast<ShapeSmem *>(smem_raw);
    const uint32_t sector = blockIdx.x;
    if (!installed[sector]) return;
    const uint32_t bds = a.band_deltas_size;
    long long *soff = reinterpret_cast<long long *>(smem_raw + sizeof(ShapeSmem));
    float *sdist = reinterpret_cast<float *>(soff + bds + 2);
    const int32_t *td = tab_deltas + (uint64_t)sector * bds;
    const float *tf = tab_dists + (uint64_t)sector * bds;
    int32_t *gdel = a.deltas + (uint64_t)sector * bds;
    float *gdist = a.dists + (uint64_t)sector * bds;
    long long last = 0;
    for (uint32_t i = threadIdx.x; i < bds; i += blockDim.x) {
        const int32_t d = td[i];
        const float x = tf[i];
        gdel[i] = d;
        gdist[i] = x;
        soff[i] = d;
        sdist[i] = x;
        if (d != 0 || __float_as_uint(x) != 0u) last = (long long)i + 1;
    }
    __syncthreads();
    sm.scan[threadIdx.x] = last;
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm.scan[threadIdx.x] = max(sm.scan[threadIdx.x], sm.scan[threadIdx.x + o]);
        __syncthreads();
    }
    const uint32_t n_filled = (uint32_t)sm.scan[0];
    __syncthreads();
    const uint32_t n_steps = n_filled + min(bds - n_filled, 2u);
    block_inclusive_scan(soff, n_filled, sm.scan);
    finish_shape(a, sector, n_filled, n_steps, 0, soff, sdist, sm);
}

// axes.rs:154-189: the f32 sight distance of every point.
__global__ void k_sight_distances(SectorTrig t, uint32_t W, uint32_t H, float *out) {
    const uint64_t n = (uint64_t)W * H;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(i / W), x = (uint32_t)(i - (uint64_t)row * W);
        out[i] = projection32(x, row_term(row, t.sight_cos), t.sight_sin);
    }
}

cudaError_t launch_sight_distances(const SectorTrig &t, uint32_t width, uint32_t height,
                                   float *out, cudaStream_t s) {
    k_sight_distances<<<148 * 4, 256, 0, s>>>(t, width, height, out);
    return cudaGetLastError();
}

size_t shape_smem_bytes() {
    return sizeof(ShapeSmem) + (size_t)(kCandidateCap + kWindowCap) * sizeof(unsigned long long);
}

cudaError_t launch_shape_tables(const ShapeArgs &a, uint32_t n_sectors, const int32_t *tab_deltas,
                                const float *tab_dists, const unsigned char *installed,
                                cudaStream_t s) {
    // the attribute is set on every launch: it belongs to the current device
    const size_t smem = shape_smem_bytes();  // covers (bds + 2) * 8 + bds * 4 (host-checked)
    cudaError_t e = cudaFuncSetAttribute(k_shape_tables, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    if (n_sectors == 0) return cudaSuccess;
    k_shape_tables<<<n_sectors, kShapeThreads, smem, s>>>(a, tab_deltas, tab_dists, installed);
    return cudaGetLastError();
}

cudaError_t launch_shape(const ShapeArgs &a, uint32_t n_sectors, cudaStream_t s) {
    // the attribute is set on every launch: it belongs to the current device
    const size_t smem = shape_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(k_shape, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    uint64_t rank_lo, rank_count;
    int axes_mode = a.sector_ids_out != nullptr;
    if (axes_mode) {
        rank_lo = a.dbg_first;
        rank_count = a.dbg_count;
    } else {
        rank_lo = (uint64_t)a.win * a.win / 2 - a.band_samples / 2;  // band_of_sight.rs:99-103
        rank_count = a.band_samples;
    }
    k_shape<<<n_sectors, kShapeThreads, smem, s>>>(a, rank_lo, rank_count, axes_mode);
    return cudaGetLastError();
}

cudaError_t launch_shape_batch(const ShapeArgs *d_args, uint32_t n_dems, uint32_t n_sectors,
                               cudaStream_t s) {
    // the attribute is set on every launch: it belongs to the current device
    const size_t smem = shape_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(k_shape_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    if (n_dems == 0 || n_sectors == 0) return cudaSuccess;
    k_shape_batch<<<n_dems * n_sectors, kShapeThreads, smem, s>>>(d_args, n_sectors);
    return cudaGetLastError();
}

}  // namespace tvs
