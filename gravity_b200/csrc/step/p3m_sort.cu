// p3m_sort.cu — cell keys, their stable radix sort, cell lists, Morton reorder.
//
// Replaces the home-cell linked lists of build_grid.comp:71-75 and the
// spatial reorder of spatial_sort_{count,scan,scatter,materials}.comp
// (GravityPipeline.kt:1269-1319).
//
// The cell lists. build_grid.comp pushes every body onto its home cell's list
// with atomicExchange, so each list's order depends on thread timing; kick.comp
// walks only the first few entries of a list (kick.comp:137-148), so that order
// changes forces. Here the order is fixed: a list runs in DESCENDING body ID,
// the order a single thread pushing IDs 0..n-1 would leave. It is produced by
// sorting the 64-bit key (cell << 32) | ~id ascending. The sort input is
// written in descending ID order, i.e. already sorted on the low 32 bits, and
// an LSD radix sort is stable, so the passes over the low 32 bits would be
// identity permutations and are skipped: only the ceil(log2 P) cell bits are
// sorted. The result is identical to sorting the full 64-bit key.
//
// The Morton reorder sorts the 32-bit tile key the same way, with ties in
// ascending ID (the reference's scatter rank is an atomic and its order inside
// a tile is nondeterministic, spatial_sort_scatter.comp:21).

#include "p3m_internal.cuh"

namespace p3m {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive warp scan.
__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t u = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim multiple of 32,
// at most 1024). `warp_tot` needs blockDim/32 entries. Returns the block total.
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot, uint32_t* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    uint32_t inc = warp_inclusive_scan(v, lane);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = lane < warps ? warp_tot[lane] : 0u;
        uint32_t ti = warp_inclusive_scan(t, lane);
        if (lane < warps) warp_tot[lane] = ti - t;
        if (lane == warps - 1) warp_tot[32] = ti;
    }
    __syncthreads();
    *out = inc - v + warp_tot[warp];
    uint32_t total = warp_tot[32];
    __syncthreads();
    return total;
}

// ----------------------------------------------------------------- scan
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanBlock = kScanThreads * kScanItems;

__device__ __forceinline__ void scan_local_body(int block, uint32_t* data, int n, uint32_t* sums) {
    __shared__ uint32_t warp_tot[33];
    const int base = block * kScanBlock + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? data[base + i] : 0u;
        s += v[i];
    }
    uint32_t pre;
    uint32_t total = block_exclusive_scan(s, warp_tot, &pre);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) data[base + i] = pre;
        pre += v[i];
    }
    if (threadIdx.x == 0 && sums) sums[block] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_local_kernel(uint32_t* data, int n,
                                                                  uint32_t* sums) {
    scan_local_body(blockIdx.x, data, n, sums);
}

__global__ void __launch_bounds__(kScanThreads) scan_add_kernel(uint32_t* data, int n,
                                                                const uint32_t* sums) {
    const uint32_t add = sums[blockIdx.x];
    const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) data[base + i] += add;
}

// ------------------------------------------------------------ radix sort

// Per-tile digit histogram, written digit-major (hist[d * tiles + tile]) so
// that one exclusive scan of the whole array yields every tile's output base
// for every digit.
__device__ __forceinline__ void radix_hist_body(int tile, const uint32_t* __restrict__ keys, int n,
                                                int shift, int bits, int tiles, uint32_t* hist) {
    __shared__ uint32_t h[kSortMaxRadix];
    const int radix = 1 << bits;
    const uint32_t mask = (uint32_t)radix - 1u;
    for (int i = threadIdx.x; i < radix; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int base = tile * kSortTile;
    // Each thread counts kSortItems consecutive keys (uint4 loads; the tile
    // base is a multiple of kSortTile keys, so every uint4 is 16-byte
    // aligned), adding a run of equal digits with one shared atomic: the
    // keys are near-sorted (cells of Morton-ordered bodies, or an earlier
    // pass's output), so runs are long.
    const int first = base + threadIdx.x * kSortItems;
    uint32_t run_digit = 0xffffffffu, run = 0;
#pragma unroll
    for (int j = 0; j < kSortItems / 4; ++j) {
        const int idx = first + j * 4;
        uint32_t k[4];
        if (idx + 3 < n) {
            uint4 q = __ldg(reinterpret_cast<const uint4*>(keys + idx));
            k[0] = q.x; k[1] = q.y; k[2] = q.z; k[3] = q.w;
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) k[e] = idx + e < n ? keys[idx + e] : 0u;
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (idx + e >= n) continue;
            const uint32_t d = (k[e] >> shift) & mask;
            if (d != run_digit) {
                if (run) atomicAdd(&h[run_digit], run);
                run_digit = d;
                run = 0;
            }
            ++run;
        }
    }
    if (run) atomicAdd(&h[run_digit], run);
    __syncthreads();
    for (int d = threadIdx.x; d < radix; d += blockDim.x) hist[(size_t)d * tiles + tile] = h[d];
}

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint32_t* __restrict__ keys,
                                                                  int n, int shift, int bits,
                                                                  int tiles, uint32_t* hist) {
    radix_hist_body(blockIdx.x, keys, n, shift, bits, tiles, hist);
}

// Look-back words: bits 31:30 say what a tile has published for a digit
// (0 nothing yet, 1 its own count, 2 its inclusive prefix over tiles), bits
// 29:0 the value. Key counts stay below 2^30.
constexpr uint32_t kLookbackAggregate = 1u << 30;
constexpr uint32_t kLookbackInclusive = 2u << 30;
constexpr uint32_t kLookbackValue = (1u << 30) - 1u;
constexpr int kLookbackWindow = 16;    // predecessors read per round trip
constexpr int kLookbackHeader = kSortMaxPasses * kLookbackMaxRadix + 32;  // totals + counters
// Header word set to 1 when a wait of this sort gave up (cleared with the
// header at the start of every look-back sort).
constexpr int kLookbackFailedWord = kSortMaxPasses * kLookbackMaxRadix + 16;

__device__ __forceinline__ uint32_t load_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void store_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Where one tile's keys go, for one digit, with decoupled look-back: the
// tiles before this one (in the order they took their indices) publish their
// counts; the sum back to the first inclusive prefix is this tile's offset.
// Every tile waited on took its index earlier, so it is running and will
// publish; each wait is still bounded (`poll_limit` polls, 200,000 unless a
// test lowers it), after which it is counted in `timeouts` and taken as 0 so
// that the kernel always ends. `status` rows are kLookbackMaxRadix words per
// tile.
__device__ __forceinline__ uint32_t lookback_exclusive(const uint32_t* status, int tile, int d,
                                                       unsigned int* timeouts, int poll_limit,
                                                       uint32_t* failed) {
    uint32_t excl = 0;
    int j = tile - 1;
    while (j >= 0) {
        uint32_t w[kLookbackWindow];
#pragma unroll
        for (int i = 0; i < kLookbackWindow; ++i)
            w[i] = j - i >= 0 ? load_relaxed(&status[(size_t)(j - i) * kLookbackMaxRadix + d])
                              : kLookbackInclusive;
#pragma unroll
        for (int i = 0; i < kLookbackWindow; ++i) {
            if (j - i < 0) return excl;
            uint32_t v = w[i];
            int spins = 0;
            while ((v & ~kLookbackValue) == 0) {
                if (++spins > poll_limit) {
                    atomicAdd(timeouts, 1u);
                    store_relaxed(failed, 1u);
                    v = kLookbackInclusive;
                    break;
                }
                __nanosleep(64);
                v = load_relaxed(&status[(size_t)(j - i) * kLookbackMaxRadix + d]);
            }
            excl += v & kLookbackValue;
            if (v & kLookbackInclusive) return excl;
        }
        j -= kLookbackWindow;
    }
    return excl;
}

// Stable scatter of one tile. Keys of warp w are the contiguous sub-tile
// [w*32*items, (w+1)*32*items), visited item-major so that (item, lane)
// increases with the input position. Each key's rank among equal digits comes
// from __match_any_sync + popc of lower lanes, plus a per-warp running count.
// The tile's output base per digit comes from the scanned tile histograms
// (LOOKBACK false), or from the pass's digit totals and a look-back over the
// tiles before it (LOOKBACK true: the tile index is taken from `counter`, and
// `hist_scanned` holds the pass's digit totals). MAXR bounds the digit count
// (2^bits); a thread handles MAXR / 256 digits where that is above 1. The
// per-warp digit counts and the tile staged in digit order share one shared
// region: each key's slot is taken from the counts before the tile is staged.
// Shared memory of one scatter tile (radix_scatter_body): the per-warp digit
// counts, then the tile staged in digit order, in one region; each digit's
// start in the tile and in the output.
template <int MAXR, int THREADS = kSortThreads>
struct ScatterShared {
    static constexpr int kWarpHist = (THREADS / 32) * MAXR;
    static constexpr int kWords = kWarpHist > 2 * kSortTile ? kWarpHist : 2 * kSortTile;
    uint32_t shared[kWords];
    uint32_t tile_start[MAXR];
    uint32_t out_base[MAXR];
    uint32_t warp_tot[33];
    int s_tile;
};

template <bool LOOKBACK, int MAXR, int THREADS = kSortThreads, int ITEMS = kSortItems>
__device__ __forceinline__ void radix_scatter_body(
    ScatterShared<MAXR, THREADS>& sm, int tile, const uint32_t* __restrict__ keys_in,
    const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, int n, int shift, int bits, int tiles,
    const uint32_t* __restrict__ hist_scanned, uint32_t* counter = nullptr,
    uint32_t* status = nullptr, unsigned int* timeouts = nullptr, int poll_limit = 0,
    int withhold_tile = -1, uint32_t* failed = nullptr) {
    constexpr int kWarps = THREADS / 32;
    constexpr int kTile = THREADS * ITEMS;
    static_assert(kTile == kSortTile, "tiles hold kSortTile keys");
    constexpr int kPer = MAXR > THREADS ? MAXR / THREADS : 1;
    uint32_t* shared = sm.shared;  // warp counts, then the staged tile
    uint32_t* tile_start = sm.tile_start;
    uint32_t* out_base = sm.out_base;
    uint32_t* warp_tot = sm.warp_tot;
    int& s_tile = sm.s_tile;
    uint32_t* warp_hist = shared;  // [warp * radix + d]
    uint32_t* s_keys = shared;
    uint32_t* s_vals = shared + kSortTile;

    if (LOOKBACK) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(counter, 1u);
        __syncthreads();
        tile = s_tile;
    }
    const int radix = 1 << bits;
    const uint32_t mask = (uint32_t)radix - 1u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile_base = tile * kSortTile;
    const int sub_base = tile_base + warp * 32 * ITEMS;
    uint32_t* my_hist = warp_hist + warp * radix;

    for (int i = threadIdx.x; i < kWarps * radix; i += blockDim.x) warp_hist[i] = 0;
    __syncthreads();

    uint32_t key[ITEMS], val[ITEMS], rank[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int idx = sub_base + j * 32 + lane;
        const bool valid = idx < n;
        key[j] = valid ? keys_in[idx] : 0u;
        val[j] = valid ? vals_in[idx] : 0u;
        const uint32_t d = valid ? (key[j] >> shift) & mask : 0xffffffffu;
        const unsigned peers = __match_any_sync(kFull, d);
        const uint32_t below = (uint32_t)__popc(peers & lanemask_lt());
        const uint32_t seen = valid ? my_hist[d] : 0u;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) my_hist[d] = seen + (uint32_t)__popc(peers);
        __syncwarp();
        rank[j] = seen + below;
    }
    __syncthreads();

    // Per digit: exclusive prefix over warps, and the tile's count; thread t
    // takes digits t*kPer .. t*kPer + kPer - 1.
    uint32_t count[kPer];
    uint32_t sum = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        count[q] = 0;
        const int d = threadIdx.x * kPer + q;
        if (d < radix) {
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const uint32_t t = warp_hist[w * radix + d];
                warp_hist[w * radix + d] = count[q];
                count[q] += t;
            }
            if (LOOKBACK && tile != withhold_tile)  // publish at once, so successors go on
                store_relaxed(&status[(size_t)tile * kLookbackMaxRadix + d],
                              (tile == 0 ? kLookbackInclusive : kLookbackAggregate) | count[q]);
            else
                out_base[d] = hist_scanned[(size_t)d * tiles + tile];
            sum += count[q];
        }
    }
    if (LOOKBACK) {
        // Start of each digit in the output: exclusive scan of the totals.
        uint32_t total = 0;
        uint32_t totals[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int d = threadIdx.x * kPer + q;
            totals[q] = d < radix ? __ldg(&hist_scanned[d]) : 0u;
            total += totals[q];
        }
        uint32_t digit_start;
        block_exclusive_scan(total, warp_tot, &digit_start);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int d = threadIdx.x * kPer + q;
            if (d < radix) {
                const uint32_t before =
                    lookback_exclusive(status, tile, d, timeouts, poll_limit, failed);
                if (tile > 0 && tile != withhold_tile)
                    store_relaxed(&status[(size_t)tile * kLookbackMaxRadix + d],
                                  kLookbackInclusive | (before + count[q]));
                out_base[d] = digit_start + before;
            }
            digit_start += totals[q];
        }
    }
    uint32_t start;
    block_exclusive_scan(sum, warp_tot, &start);
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const int d = threadIdx.x * kPer + q;
        if (d < radix) tile_start[d] = start;
        start += count[q];
    }
    __syncthreads();

    // Each key's slot in the tile staged in digit order.
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int idx = sub_base + j * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[j] >> shift) & mask;
            rank[j] += tile_start[d] + my_hist[d];
        }
    }
    __syncthreads();  // the counts are read; their space becomes the staged tile
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int idx = sub_base + j * 32 + lane;
        if (idx < n) {
            s_keys[rank[j]] = key[j];
            s_vals[rank[j]] = val[j];
        }
    }
    __syncthreads();

    // Write the tile back in digit order: consecutive threads write
    // consecutive addresses inside each digit's run.
    const int tile_n = min(kSortTile, n - tile_base);
    for (int p = threadIdx.x; p < tile_n; p += blockDim.x) {
        const uint32_t k = s_keys[p];
        const uint32_t d = (k >> shift) & mask;
        const uint32_t o = out_base[d] + ((uint32_t)p - tile_start[d]);
        keys_out[o] = k;
        vals_out[o] = s_vals[p];
    }
}

__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int n, int shift, int bits,
    int tiles, const uint32_t* __restrict__ hist_scanned) {
    __shared__ ScatterShared<kSortMaxRadix> sm;
    radix_scatter_body<false, kSortMaxRadix>(sm, blockIdx.x, keys_in, vals_in, keys_out, vals_out,
                                             n, shift, bits, tiles, hist_scanned);
}

// One pass of the one-kernel-per-pass sort: `totals` = this pass's digit
// totals, `status` = this pass's [tiles][kLookbackMaxRadix] look-back words.
// MAXR: 256 for 8-bit digits, 512 for 9-bit ones.
// 512 threads of 8 keys each: a sort of a few hundred thousand keys has one
// tile per SM, and twice the warps hide more of each tile's latency.
constexpr int kLookbackThreads = 512;
constexpr int kLookbackItems = kSortTile / kLookbackThreads;

template <int MAXR>
__global__ void __launch_bounds__(kLookbackThreads) lookback_scatter_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int n, int shift, int bits,
    int tiles, const uint32_t* __restrict__ totals, uint32_t* counter, uint32_t* status,
    unsigned int* timeouts, int poll_limit, int withhold_tile, uint32_t* failed) {
    grid_dependency_wait();
    __shared__ ScatterShared<MAXR, kLookbackThreads> sm;
    radix_scatter_body<true, MAXR, kLookbackThreads, kLookbackItems>(
        sm, 0, keys_in, vals_in, keys_out, vals_out, n, shift, bits, tiles, totals, counter,
        status, timeouts, poll_limit, withhold_tile, failed);
}

// Digit totals of every pass in one read of the keys: per-CTA shared counts
// (runs of equal digits added at once, as in radix_hist_body), then one global
// atomic per CTA and digit. totals[p * kLookbackMaxRadix + d] must start at
// zero.
__global__ void __launch_bounds__(kSortThreads) lookback_totals_kernel(
    const uint32_t* __restrict__ keys, int n, int passes, int bits, int key_bits,
    uint32_t* totals) {
    grid_dependency_wait();
    __shared__ uint32_t h[kSortMaxPasses][kLookbackMaxRadix];
    for (int i = threadIdx.x; i < kSortMaxPasses * kLookbackMaxRadix; i += blockDim.x)
        (&h[0][0])[i] = 0;
    __syncthreads();
    uint32_t run_digit[kSortMaxPasses], run[kSortMaxPasses], mask[kSortMaxPasses];
#pragma unroll
    for (int p = 0; p < kSortMaxPasses; ++p) {
        run_digit[p] = 0xffffffffu;
        run[p] = 0;
        const int pb = min(bits, key_bits - p * bits);
        mask[p] = pb > 0 ? (1u << pb) - 1u : 0u;
    }
    for (int base = blockIdx.x * kSortTile; base < n; base += gridDim.x * kSortTile) {
        const int first = base + threadIdx.x * kSortItems;
#pragma unroll
        for (int j = 0; j < kSortItems / 4; ++j) {
            const int idx = first + j * 4;
            uint32_t k[4];
            if (idx + 3 < n) {
                const uint4 q = __ldg(reinterpret_cast<const uint4*>(keys + idx));
                k[0] = q.x; k[1] = q.y; k[2] = q.z; k[3] = q.w;
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) k[e] = idx + e < n ? keys[idx + e] : 0u;
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                if (idx + e >= n) continue;
#pragma unroll
                for (int p = 0; p < kSortMaxPasses; ++p) {
                    if (p >= passes) break;
                    const uint32_t d = (k[e] >> (p * bits)) & mask[p];
                    if (d != run_digit[p]) {
                        if (run[p]) atomicAdd(&h[p][run_digit[p]], run[p]);
                        run_digit[p] = d;
                        run[p] = 0;
                    }
                    ++run[p];
                }
            }
        }
    }
#pragma unroll
    for (int p = 0; p < kSortMaxPasses; ++p)
        if (p < passes && run[p]) atomicAdd(&h[p][run_digit[p]], run[p]);
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kLookbackMaxRadix; i += blockDim.x) {
        const uint32_t v = (&h[0][0])[i];
        if (v) atomicAdd(&totals[i], v);
    }
}

// ----------------------------------------------------------- key kernels
// build_grid.comp:71-72: home = ivec2(floor(p * vec2(W, H))), then wrapCell.
__device__ __forceinline__ uint32_t home_cell(float x, float y, int W, int H) {
    const int hx = wrap_index(float_to_int(floorf(__fmul_rn(x, (float)W))), W);
    const int hy = wrap_index(float_to_int(floorf(__fmul_rn(y, (float)H))), H);
    return (uint32_t)hx + (uint32_t)hy * (uint32_t)W;
}

__global__ void cell_keys_kernel(const float4* __restrict__ bodies, int n, int W, int H,
                                 uint32_t* keys, uint32_t* vals) {
    grid_dependency_wait();
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const float4 b = bodies[id];
    const int slot = n - 1 - id;  // descending ID order
    keys[slot] = home_cell(b.x, b.y, W, H);
    vals[slot] = (uint32_t)id;
}

// spatial_sort_key.glsl:7-25.
__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__device__ __forceinline__ uint32_t tile_coord(float p, int size) {
    // floor then clamp; NaN maps to tile 0, +-inf to the clamp limits.
    const float f = floorf(__fmul_rn(p, (float)size));
    int t;
    if (f != f) t = 0;
    else if (f >= 2147483647.0f) t = 2147483647;
    else if (f <= -2147483648.0f) t = (int)0x80000000;
    else t = (int)f;
    return (uint32_t)min(max(t, 0), size - 1);
}

__device__ __forceinline__ uint32_t morton_key(float4 b, int wbits, int hbits) {
    const uint32_t tx = tile_coord(b.x, 1 << wbits), ty = tile_coord(b.y, 1 << hbits);
    const int common = min(wbits, hbits);
    const uint32_t low = (1u << common) - 1u;
    const uint32_t morton = spread_bits(tx & low) | (spread_bits(ty & low) << 1);
    return morton | (((tx | ty) >> common) << (2 * common));
}

__device__ __forceinline__ void morton_keys_body(int block, const float4* __restrict__ bodies, int n,
                                                 int wbits, int hbits, uint32_t* keys,
                                                 uint32_t* vals) {
    const int id = block * blockDim.x + threadIdx.x;
    if (id >= n) return;
    keys[id] = morton_key(bodies[id], wbits, hbits);
    vals[id] = (uint32_t)id;
}

// The Morton keys, and (totals.totals set) their digit totals for the
// look-back sort that follows.
__global__ void morton_keys_kernel(const float4* __restrict__ bodies, int n, int wbits, int hbits,
                                   uint32_t* keys, uint32_t* vals, SortTotals totals) {
    grid_dependency_wait();
    if (!totals.totals) {
        morton_keys_body(blockIdx.x, bodies, n, wbits, hbits, keys, vals);
        return;
    }
    __shared__ uint32_t sh[kSortMaxPasses * kLookbackMaxRadix];
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = id < n;
    uint32_t key = 0;
    if (valid) {
        key = morton_key(bodies[id], wbits, hbits);
        keys[id] = key;
        vals[id] = (uint32_t)id;
    }
    add_digit_totals(totals, valid, key, sh);
}

// spatial_sort_scatter.comp:14-28 and spatial_sort_materials.comp:9-13: a
// bit-for-bit permutation; destinations[src] = new ID.
__device__ __forceinline__ void permute_body(int block, const uint32_t* __restrict__ order, int n,
                                             const float4* __restrict__ bodies,
                                             const float2* __restrict__ accel,
                                             const float4* __restrict__ materials,
                                             float4* bodies_out, float2* accel_out,
                                             float4* materials_out, uint32_t* destinations,
                                             bool identity = false) {
    const int t = block * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t src = identity ? (uint32_t)t : order[t];
    bodies_out[t] = bodies[src];
    accel_out[t] = accel[src];
    materials_out[t] = materials[src];
    destinations[src] = (uint32_t)t;
}

__global__ void permute_kernel(const uint32_t* __restrict__ order, int n,
                               const float4* __restrict__ bodies, const float2* __restrict__ accel,
                               const float4* __restrict__ materials, float4* bodies_out,
                               float2* accel_out, float4* materials_out, uint32_t* destinations,
                               const uint32_t* __restrict__ sort_failed) {
    grid_dependency_wait();
    const bool identity = sort_failed != nullptr && *sort_failed != 0u;
    permute_body(blockIdx.x, order, n, bodies, accel, materials, bodies_out, accel_out,
                 materials_out, destinations, identity);
}

// Cell lists from the sorted keys. Run starts write cell_start; counts and
// the fixed-point cell masses (build_grid.comp:74-75) are reduced over each
// warp's segment of equal keys, then added with one atomic per segment
// (integer sums, so the result does not depend on the order).
// The whole warp stores value v into cell_start[f0, f1) for every lane's
// range, one lane's range after another (gaps can be long when cells far
// outnumber bodies).
__device__ __forceinline__ void fill_ranges(int* cell_start, uint32_t f0, uint32_t f1, int v) {
    const int lane = threadIdx.x & 31;
    unsigned pending = __ballot_sync(kFull, f1 > f0);
    while (pending) {
        const int src = __ffs(pending) - 1;
        pending &= pending - 1;
        const uint32_t a = __shfl_sync(kFull, f0, src), b = __shfl_sync(kFull, f1, src);
        const int value = __shfl_sync(kFull, v, src);
        for (uint32_t c = a + lane; c < b; c += 32) cell_start[c] = value;
    }
}

// One sorted entry of the cell build: its cell key and the keys either side
// (equal keys are contiguous lanes), its body's ID, position and mass.
struct BuildItem {
    int i;
    bool valid;
    uint32_t c, prev, next, id;
    float4 b;
    float m;
};

// The entry's key, its neighbours' keys (shuffles, and one load at each end
// of the warp) and its ID: entry i of a warp-contiguous run of 32.
__device__ __forceinline__ void build_load_keys(BuildItem& it, int i, const uint32_t* __restrict__ keys,
                                                const uint32_t* __restrict__ ids, int n) {
    const int lane = threadIdx.x & 31;
    it.i = i;
    it.valid = i < n;
    it.c = it.valid ? keys[i] : 0xffffffffu;
    it.prev = __shfl_up_sync(kFull, it.c, 1);
    if (lane == 0) it.prev = (it.valid && i > 0) ? keys[i - 1] : 0xfffffffeu;
    it.next = __shfl_down_sync(kFull, it.c, 1);
    if (lane == 31) it.next = (i + 1 < n) ? keys[i + 1] : 0xfffffffeu;
    it.id = it.valid ? ids[i] : 0u;
}

// The body's position and mass (the ID-ordered gathers).
__device__ __forceinline__ void build_gather(BuildItem& it, const float4* __restrict__ bodies,
                                             const float4* __restrict__ materials) {
    if (it.valid) {
        it.b = bodies[it.id];
        it.m = materials[it.id].x;
    }
}

// The entry, the run's count and mass (segmented sum across the warp, one
// atomic per run and warp), the run's start, and (fill_cells > 0) the starts
// of the empty cells.
__device__ __forceinline__ void build_finish(const BuildItem& it, int n, int* cell_start,
                                             int* cell_count, uint32_t* cell_mass, float4* entries,
                                             int fill_cells) {
    const int lane = threadIdx.x & 31;
    const int i = it.i;
    const uint32_t c = it.c, prev = it.prev, next = it.next;
    const bool valid = it.valid;
    uint32_t cnt = 0, mq = 0;
    if (valid) {
        entries[i] = make_float4(it.b.x, it.b.y, it.m, __uint_as_float(it.id));
        cnt = 1;
        mq = (uint32_t)__float2uint_rn(__fmul_rn(it.m, kCellMassUnits));
        if (i == 0 || prev != c) cell_start[c] = i;
    }
    // Segmented inclusive sum over equal keys (keys are sorted, so equal keys
    // are contiguous lanes).
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t oc = __shfl_up_sync(kFull, cnt, o);
        const uint32_t om = __shfl_up_sync(kFull, mq, o);
        const uint32_t ok = __shfl_up_sync(kFull, c, o);
        if (lane >= o && ok == c) {
            cnt += oc;
            mq += om;
        }
    }
    const bool tail = valid && (lane == 31 || next != c);
    if (tail) {
        atomicAdd(&cell_count[c], (int)cnt);
        atomicAdd(&cell_mass[c], mq);
    }
    if (fill_cells > 0) {
        // Full CSR: an empty cell starts where the next occupied cell does,
        // and cell_start[fill_cells] = n. The head of each run fills the
        // empty cells before it; the last entry fills the cells after it.
        const bool head = valid && (i == 0 || prev != c);
        const uint32_t g0 = (i == 0) ? 0u : prev + 1u;
        fill_ranges(cell_start, head ? g0 : 0u, head ? c : 0u, i);
        const bool last = valid && i == n - 1;
        fill_ranges(cell_start, last ? c + 1u : 0u, last ? (uint32_t)fill_cells + 1u : 0u, n);
    }
}

// Each warp takes kCellBuildItems runs of 32 consecutive entries and issues
// all their gathers before it uses the first, so twice the gathers are in
// flight: block b of 256 threads covers entries [512 b, 512 b + 512).
__device__ __forceinline__ void cell_build_body(int block, const uint32_t* __restrict__ keys,
                                                const uint32_t* __restrict__ ids, int n,
                                                const float4* __restrict__ bodies,
                                                const float4* __restrict__ materials,
                                                int* cell_start, int* cell_count,
                                                uint32_t* cell_mass, float4* entries,
                                                int fill_cells) {
    const int warp_base =
        (block * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 * kCellBuildItems);
    BuildItem it[kCellBuildItems];
#pragma unroll
    for (int j = 0; j < kCellBuildItems; ++j)
        build_load_keys(it[j], warp_base + 32 * j + (threadIdx.x & 31), keys, ids, n);
#pragma unroll
    for (int j = 0; j < kCellBuildItems; ++j) build_gather(it[j], bodies, materials);
#pragma unroll
    for (int j = 0; j < kCellBuildItems; ++j)
        build_finish(it[j], n, cell_start, cell_count, cell_mass, entries, fill_cells);
}

__global__ void cell_build_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ ids,
                                  int n, const float4* __restrict__ bodies,
                                  const float4* __restrict__ materials, int* cell_start,
                                  int* cell_count, uint32_t* cell_mass, float4* entries,
                                  int fill_cells, const uint32_t* __restrict__ sort_failed) {
    grid_dependency_wait();
    // A sort whose look-back gave up leaves keys and IDs that are not a
    // permutation: build nothing (every cell stays empty).
    if (sort_failed != nullptr && *sort_failed != 0u) return;
    cell_build_body(blockIdx.x, keys, ids, n, bodies, materials, cell_start, cell_count, cell_mass,
                    entries, fill_cells);
}

// ------------------------------------------------------- batched launches
__global__ void __launch_bounds__(kSortThreads) radix_hist_batched_kernel(
    const RadixArgs* __restrict__ args, const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const RadixArgs a = args[sb.x];
    radix_hist_body(sb.y, a.keys_in, a.n, a.shift, a.bits, a.tiles, a.hist);
}

// The look-back scatter's CTA shape (512 threads of 8 keys: 64 registers,
// twice the warps per SM of 256 threads of 16 keys at 127 registers) on
// the same 4096-key tiles; a stable sort's output does not depend on it.
__global__ void __launch_bounds__(kLookbackThreads) radix_scatter_batched_kernel(
    const RadixArgs* __restrict__ args, const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const RadixArgs a = args[sb.x];
    __shared__ ScatterShared<kSortMaxRadix, kLookbackThreads> sm;
    radix_scatter_body<false, kSortMaxRadix, kLookbackThreads, kLookbackItems>(
        sm, sb.y, a.keys_in, a.vals_in, a.keys_out, a.vals_out, a.n, a.shift, a.bits, a.tiles,
        a.hist);
}

__global__ void __launch_bounds__(kScanThreads) scan_batched_kernel(
    const ScanArgs* __restrict__ args, const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const ScanArgs a = args[sb.x];
    scan_local_body(0, a.data, a.n, nullptr);
}

__global__ void morton_keys_batched_kernel(const MortonArgs* __restrict__ args,
                                           const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const MortonArgs a = args[sb.x];
    morton_keys_body(sb.y, a.bodies, a.n, a.wbits, a.hbits, a.keys, a.vals);
}

__global__ void permute_batched_kernel(const PermuteArgs* __restrict__ args,
                                       const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const PermuteArgs a = args[sb.x];
    permute_body(sb.y, a.order, a.n, a.bodies, a.accel, a.materials, a.bodies_out, a.accel_out,
                 a.materials_out, a.destinations);
}

__global__ void cell_build_batched_kernel(const CellBuildArgs* __restrict__ args,
                                          const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const CellBuildArgs a = args[sb.x];
    cell_build_body(sb.y, a.keys, a.ids, a.n, a.bodies, a.materials, a.cell_start, a.cell_count,
                    a.cell_mass, a.entries, 0);
}

// Zeroes `words` 32-bit words per simulation; local block b takes words
// [b * 1024 * 4, ...) as uint4 where aligned.
__global__ void zero_batched_kernel(const ZeroArgs* __restrict__ args,
                                    const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const ZeroArgs a = args[sb.x];
    const long long base = (long long)sb.y * (kBatchThreads * 16);
    for (int i = threadIdx.x; i < kBatchThreads * 16; i += blockDim.x) {
        const long long w = base + i;
        if (w < a.words) a.data[w] = 0u;
    }
}

inline int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace

// Host-side launchers: not part of the coherent copy of the bodies that the
// batched form's persistent kernel uses (p3m_step.cu).
#ifndef P3M_COHERENT_BODIES

size_t sort_hist_entries(int capacity) {
    const size_t tiles = ((size_t)capacity + kSortTile - 1) / kSortTile;
    return (size_t)kSortMaxRadix * (tiles > 0 ? tiles : 1);
}

size_t sort_lookback_words(int capacity) {
    const size_t tiles = ((size_t)capacity + kSortTile - 1) / kSortTile;
    return (size_t)kLookbackHeader +
           (size_t)kSortMaxPasses * (tiles > 0 ? tiles : 1) * kLookbackMaxRadix;
}

size_t sort_block_sum_entries(int capacity) {
    const size_t h = sort_hist_entries(capacity);
    return (h + kScanBlock - 1) / kScanBlock + 1;
}

cudaError_t exclusive_scan_u32(uint32_t* data, int n, uint32_t* block_sums, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int blocks = blocks_for(n, kScanBlock);
    if (blocks == 1) {
        scan_local_kernel<<<1, kScanThreads, 0, stream>>>(data, n, nullptr);
        count_launches(1);
        return cudaGetLastError();
    }
    if (blocks > kScanBlock) return cudaErrorInvalidValue;
    scan_local_kernel<<<blocks, kScanThreads, 0, stream>>>(data, n, block_sums);
    scan_local_kernel<<<1, kScanThreads, 0, stream>>>(block_sums, blocks, nullptr);
    scan_add_kernel<<<blocks, kScanThreads, 0, stream>>>(data, n, block_sums);
    count_launches(3);
    return cudaGetLastError();
}

// Passes and digit width of the look-back form, or false when a sort of n
// keys does not take it. With no per-pass histogram or scan to pay for,
// 9-bit digits are used where they save a pass (17 or 18 key bits: 2 passes
// instead of 3).
static bool lookback_plan(const SortScratch& s, int n, int key_bits, int* passes, int* bits) {
    int p = (key_bits + 7) / 8;
    if (!s.lookback || !s.wait_timeouts || n <= 1 || n >= (1 << 30) || key_bits <= 0 ||
        p > kSortMaxPasses)
        return false;
    if (p > 1 && (key_bits + 8) / 9 < p) p = (key_bits + 8) / 9;
    *passes = p;
    *bits = (key_bits + p - 1) / p;
    return true;
}

static size_t lookback_words(int n, int passes) {
    return (size_t)kLookbackHeader + (size_t)passes * blocks_for(n, kSortTile) * kLookbackMaxRadix;
}

// Below this many keys the producer adds the digit totals: the separate
// totals kernel's launch is then the larger cost. Above it, a producer CTA's
// per-pass bins and the global atomics on shared high digits cost more than
// one streaming read of the keys.
constexpr int kProducerTotalsMaxKeys = 1 << 21;

cudaError_t radix_sort_prepare(const SortScratch& s, int n, int key_bits, cudaStream_t stream,
                               SortTotals* out) {
    *out = SortTotals();
    int passes, bits;
    if (n > s.capacity || n >= kProducerTotalsMaxKeys ||
        !lookback_plan(s, n, key_bits, &passes, &bits))
        return cudaSuccess;
    cudaError_t e =
        cudaMemsetAsync(s.lookback, 0, lookback_words(n, passes) * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    out->totals = s.lookback;
    out->passes = passes;
    out->bits = bits;
    out->key_bits = key_bits;
    return cudaSuccess;
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, const SortScratch& s, int n,
                             int key_bits, cudaStream_t stream, uint32_t** out_keys,
                             uint32_t** out_vals, bool totals_ready, const uint32_t** failed) {
    *out_keys = keys;
    *out_vals = vals;
    if (failed) *failed = nullptr;
    if (n <= 1 || key_bits <= 0) return cudaSuccess;
    if (n > s.capacity) return cudaErrorInvalidValue;
    const int passes = (key_bits + 7) / 8;
    const int bits = (key_bits + passes - 1) / passes;
    const int tiles = blocks_for(n, kSortTile);
    uint32_t* kin = keys;
    uint32_t* vin = vals;
    uint32_t* kout = s.keys_alt;
    uint32_t* vout = s.vals_alt;
    int lb_passes, lb_bits;
    if (lookback_plan(s, n, key_bits, &lb_passes, &lb_bits)) {
        uint32_t* failed_word = s.lookback + kLookbackFailedWord;
        if (failed) *failed = failed_word;
        // One kernel per pass: the digit totals of all passes first (here, or
        // by the keys' producer after radix_sort_prepare), then each pass's
        // tiles find their offsets by look-back.
        if (!totals_ready) {
            cudaError_t e = cudaMemsetAsync(s.lookback, 0,
                                            lookback_words(n, lb_passes) * sizeof(uint32_t), stream);
            if (e != cudaSuccess) return e;
            const int tblocks = min(tiles, 4 * 148);
            launch_chained(lookback_totals_kernel, tblocks, kSortThreads, 0, stream, kin, n,
                           lb_passes, lb_bits, key_bits, s.lookback);
            count_launches(1);
        }
        for (int p = 0; p < lb_passes; ++p) {
            const int shift = p * lb_bits;
            const int pbits = min(lb_bits, key_bits - shift);
            const uint32_t* totals = s.lookback + p * kLookbackMaxRadix;
            uint32_t* counter = s.lookback + kSortMaxPasses * kLookbackMaxRadix + p;
            uint32_t* status = s.lookback + kLookbackHeader + (size_t)p * tiles * kLookbackMaxRadix;
            if (pbits > 8)
                launch_chained(lookback_scatter_kernel<512>, tiles, kLookbackThreads, 0, stream,
                    kin, vin, kout, vout, n, shift, pbits, tiles, totals, counter, status,
                    s.wait_timeouts, s.poll_limit, s.withhold_tile, failed_word);
            else
                launch_chained(lookback_scatter_kernel<256>, tiles, kLookbackThreads, 0, stream,
                    kin, vin, kout, vout, n, shift, pbits, tiles, totals, counter, status,
                    s.wait_timeouts, s.poll_limit, s.withhold_tile, failed_word);
            count_launches(1);
            uint32_t* tk = kin; kin = kout; kout = tk;
            uint32_t* tv = vin; vin = vout; vout = tv;
        }
        *out_keys = kin;
        *out_vals = vin;
        return cudaGetLastError();
    }
    for (int p = 0; p < passes; ++p) {
        const int shift = p * bits;
        const int pbits = min(bits, key_bits - shift);
        radix_hist_kernel<<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, pbits, tiles, s.hist);
        cudaError_t e = exclusive_scan_u32(s.hist, (1 << pbits) * tiles, s.block_sums, stream);
        if (e != cudaSuccess) return e;
        radix_scatter_kernel<<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, shift,
                                                                 pbits, tiles, s.hist);
        count_launches(2);
        uint32_t* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
    }
    *out_keys = kin;
    *out_vals = vin;
    return cudaGetLastError();
}

cudaError_t launch_cell_keys(const float4* bodies, int n, GridShape g, uint32_t* keys,
                             uint32_t* vals, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    launch_chained(cell_keys_kernel, blocks_for(n, 256), 256, 0, stream, bodies, n, g.W, g.H, keys, vals);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_morton_keys(const float4* bodies, int n, int wbits, int hbits, uint32_t* keys,
                               uint32_t* vals, cudaStream_t stream, SortTotals totals) {
    if (n <= 0) return cudaSuccess;
    launch_chained(morton_keys_kernel, blocks_for(n, 256), 256, 0, stream, bodies, n, wbits, hbits,
                   keys, vals, totals);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_permute(const uint32_t* order, int n, const float4* bodies, const float2* accel,
                           const float4* materials, float4* bodies_out, float2* accel_out,
                           float4* materials_out, uint32_t* destinations, cudaStream_t stream,
                           const uint32_t* sort_failed) {
    if (n <= 0) return cudaSuccess;
    launch_chained(permute_kernel, blocks_for(n, 256), 256, 0, stream, order, n, bodies, accel, materials,
                                                           bodies_out, accel_out, materials_out,
                                                           destinations, sort_failed);
    count_launches(1);
    return cudaGetLastError();
}

int radix_tiles(int n) { return blocks_for(n, kSortTile); }
int radix_scan_limit() { return kScanBlock; }

#define P3M_BATCHED(name, Args, kernel, threads)                                \
    cudaError_t name(const Args* a, BatchGrid g, cudaStream_t s) {            \
        if (g.blocks <= 0) return cudaSuccess;                                 \
        kernel<<<g.blocks, threads, 0, s>>>(a, g.first, g.sims);               \
        count_launches(1);                                                     \
        return cudaGetLastError();                                             \
    }
P3M_BATCHED(batched_morton_keys, MortonArgs, morton_keys_batched_kernel, kBatchThreads)
P3M_BATCHED(batched_radix_hist, RadixArgs, radix_hist_batched_kernel, kSortThreads)
P3M_BATCHED(batched_scan, ScanArgs, scan_batched_kernel, kScanThreads)
P3M_BATCHED(batched_radix_scatter, RadixArgs, radix_scatter_batched_kernel, kLookbackThreads)
P3M_BATCHED(batched_permute, PermuteArgs, permute_batched_kernel, kBatchThreads)
P3M_BATCHED(batched_cell_build, CellBuildArgs, cell_build_batched_kernel, kBatchThreads)
P3M_BATCHED(batched_zero, ZeroArgs, zero_batched_kernel, kBatchThreads)
#undef P3M_BATCHED

cudaError_t launch_cell_build(const uint32_t* keys, const uint32_t* ids, int n, const float4* bodies,
                              const float4* materials, int* cell_start, int* cell_count,
                              uint32_t* cell_mass, float4* entries, int fill_cells,
                              cudaStream_t stream, const uint32_t* sort_failed) {
    if (n <= 0) {
        if (fill_cells > 0)
            return cudaMemsetAsync(cell_start, 0, ((size_t)fill_cells + 1) * sizeof(int), stream);
        return cudaSuccess;
    }
    launch_chained(cell_build_kernel, blocks_for(n, kCellBuildBlockEntries), 256, 0, stream, keys, ids, n, bodies, materials,
                                                              cell_start, cell_count, cell_mass,
                                                              entries, fill_cells, sort_failed);
    count_launches(1);
    return cudaGetLastError();
}

#endif  // !P3M_COHERENT_BODIES
}  // namespace p3m
