// p3m_deposit.cu — CIC mass deposit by mesh tiles that own their cells.
//
// Restates build_grid.comp:53-69: each body spreads mass * CIC weight over the
// four mesh cells around p * (W, H) - 0.5, as fixed-point integers, with the
// mesh wrap of wrapMesh (build_grid.comp:29-42). Integer sums commute, so the
// grid is bit-identical whatever the order of the additions.
//
// Two kernels. Below kTileMinBodies bodies, CTAs take chunks of the cell
// order (deposit_chunks_kernel, below). From there on, mesh tiles own their
// cells:
//
// One CTA owns a TX x TY tile of the mesh. A body deposits into
// mesh columns bx, bx+1 with bx = hx - 1 or hx (hx its home column), so the
// bodies that reach the tile live in home columns [c0-1, c0+TX] and home rows
// [r0-1, r0+TY] (taken modulo the mesh, and kept where they are physical
// cells). The bodies arrive in cell order and cell_start is a full CSR, so
// each of those TY+2 home rows is one or two contiguous runs of entries found
// with two loads. The CTA accumulates the corners that land in its tile in
// shared memory and stores the tile with plain coalesced stores: no global
// atomics, no clearing pass, each mesh cell written once.
//
// A tile denser than kDenseBodiesPerCell bodies per cell sums its bodies per
// home cell in registers first (dense cells would otherwise serialise on a
// few shared addresses). A tile with more than
// kTileCap bodies (a cluster) would leave its CTA far behind the others; it
// stores zeros instead and queues its bodies in pieces of kPiece,
// which a second, persistent kernel spreads over all SMs and adds with
// global atomics (the tile is zero by then: stream order). The int64 form
// accumulates in 32-bit shared words with an explicit carry word, a native
// shared atomic instead of a 64-bit compare-and-swap loop.
//
// Arithmetic is written with explicit round-to-nearest intrinsics so that no
// multiply-add is contracted: the weights must round exactly as the oracle's.

#include <climits>

#include "p3m_internal.cuh"

namespace p3m {
namespace {

constexpr int kThreads = 256;
constexpr int kTileX = 256, kTileY = 16;  // at most; smaller meshes use the mesh size
constexpr int kMaxRuns = 2 * (kTileY + 2);
// tile_runs takes one lane of warp 0 per home row (TY + 2 of them) and
// writes runs 2*lane and 2*lane + 1: every run slot is written only while
// the home rows fit one warp.
static_assert(kTileY + 2 <= 32, "tile_runs needs one lane per home row");
constexpr int kTileCap = 16384;  // bodies a tile takes alone
constexpr int kPiece = 2048;    // entries per piece of a heavy tile
// Below this many bodies the entry-chunk kernel is used: a small mesh has
// too few tiles to fill the GPU and clustering would unbalance them.
constexpr int kTileMinBodies = 1 << 21;

template <typename T>
__device__ __forceinline__ T quantize(float w, float scale);
template <>
__device__ __forceinline__ uint32_t quantize<uint32_t>(float w, float scale) {
    return __float2uint_rn(__fmul_rn(w, scale));  // uint(round(w * massScale))
}
template <>
__device__ __forceinline__ unsigned long long quantize<unsigned long long>(float w, float scale) {
    // int64 form: 2^-32 mass quanta; scale = 2^32 exactly. Values are
    // non-negative, so two's-complement int64 sums equal these unsigned sums.
    return (unsigned long long)__float2ll_rn(__fmul_rn(w, scale));
}

struct TileGeom {
    int W, H, MW, MH, TX, TY, tiles_x;
    int tx_log2;  // TX is a power of two
};

// The runs of entries whose bodies can reach tile `tile`, in shared memory;
// returns their total length. Warp 0 computes them; ends with a barrier.
__device__ int tile_runs(const int* __restrict__ cell_start, const TileGeom& g, int tile,
                         int* run_begin, int* run_end, int* run_prefix, int* s_total) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const int c0 = (tile % g.tiles_x) * g.TX, r0 = (tile / g.tiles_x) * g.TY;
        const bool all_cols = g.TX == g.MW, all_rows = g.TY == g.MH;
        const int nrows = all_rows ? g.MH : g.TY + 2;
        int b0 = 0, e0 = 0, b1 = 0, e1 = 0;
        if (lane < nrows) {
            const int m = all_rows ? lane : r0 - 1 + lane;
            const int hr = m < 0 ? m + g.MH : (m >= g.MH ? m - g.MH : m);
            if (hr < g.H) {
                // Home columns [a, b] in mesh space, split where they wrap,
                // clipped to the physical columns.
                int a0, a1, a2 = 0, a3 = -1;
                if (all_cols) { a0 = 0; a1 = g.MW - 1; }
                else {
                    a0 = c0 - 1; a1 = c0 + g.TX;
                    if (a0 < 0) { a2 = g.MW - 1; a3 = g.MW - 1; a0 = 0; }
                    else if (a1 >= g.MW) { a2 = 0; a3 = 0; a1 = g.MW - 1; }
                }
                const int row = hr * g.W;
                auto run = [&](int a, int b, int& rb, int& re) {
                    if (b >= g.W) b = g.W - 1;
                    if (a > b) return;
                    rb = __ldg(&cell_start[row + a]);
                    re = __ldg(&cell_start[row + b + 1]);
                };
                run(a0, a1, b0, e0);
                if (a3 >= a2) run(a2, a3, b1, e1);
            }
        }
        // Runs 2*lane and 2*lane+1; inclusive prefix of their lengths.
        const int len = (e0 - b0) + (e1 - b1);
        int inc = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane < kMaxRuns / 2) {
            run_begin[2 * lane] = b0;
            run_end[2 * lane] = e0;
            run_begin[2 * lane + 1] = b1;
            run_end[2 * lane + 1] = e1;
            run_prefix[2 * lane] = inc - len;           // start of run 2*lane
            run_prefix[2 * lane + 1] = inc - len + (e0 - b0);
        }
        if (lane == 31) *s_total = inc;
    }
    __syncthreads();
    return *s_total;
}

// Tile accumulators: 32-bit words; the int64 form keeps a high word per cell
// and carries into it (a native 32-bit shared atomic instead of a 64-bit one).
template <typename T>
struct TileAcc;
// The split form (sparse tiles, add_split / get_split) adds without reading
// back: a 32-bit value as it is, a 64-bit value q as a high part into hi and
// the rest (at most 2^19) into lo, value = hi * 2^19 + lo, two shared
// atomics whose results are not waited for. Exact while a cell gets at most
// 8191 additions of values below 2^38 (each word's sum stays below 2^32): a
// sparse tile holds fewer than 8192 bodies, and a tile that meets a larger
// value (a body of mass 64 or more) is redone with the carry form.
constexpr int kSplitShift = 19;
constexpr unsigned long long kSplitMax = 1ull << 38;

template <>
struct TileAcc<uint32_t> {
    uint32_t lo[kTileX * kTileY];
    __device__ __forceinline__ void zero(int i) { lo[i] = 0u; }
    __device__ __forceinline__ void add(int i, uint32_t v) {
        if (v) atomicAdd(&lo[i], v);
    }
    __device__ __forceinline__ uint32_t get(int i) const { return lo[i]; }
    __device__ __forceinline__ void add_split(int i, uint32_t v) { atomicAdd(&lo[i], v); }
    __device__ __forceinline__ uint32_t get_split(int i) const { return lo[i]; }
    __device__ __forceinline__ static bool too_large(uint32_t) { return false; }
};
template <>
struct TileAcc<unsigned long long> {
    uint32_t lo[kTileX * kTileY];
    uint32_t hi[kTileX * kTileY];
    __device__ __forceinline__ void zero(int i) { lo[i] = 0u; hi[i] = 0u; }
    __device__ __forceinline__ void add(int i, unsigned long long v) {
        const uint32_t vl = (uint32_t)v;
        uint32_t vh = (uint32_t)(v >> 32);
        if (vl) {
            const uint32_t old = atomicAdd(&lo[i], vl);
            vh += (old > 0xffffffffu - vl) ? 1u : 0u;  // carry out of the low word
        }
        if (vh) atomicAdd(&hi[i], vh);
    }
    __device__ __forceinline__ unsigned long long get(int i) const {
        return ((unsigned long long)hi[i] << 32) | lo[i];
    }
    __device__ __forceinline__ void add_split(int i, unsigned long long v) {
        atomicAdd(&lo[i], (uint32_t)v & ((1u << kSplitShift) - 1u));
        atomicAdd(&hi[i], (uint32_t)(v >> kSplitShift));
    }
    __device__ __forceinline__ unsigned long long get_split(int i) const {
        return ((unsigned long long)hi[i] << kSplitShift) + lo[i];
    }
    __device__ __forceinline__ static bool too_large(unsigned long long v) {
        return v >= kSplitMax;
    }
};

// Clears the accumulator planes of `cells` cells (a multiple of 16) with
// 16-byte stores.
template <typename T>
__device__ __forceinline__ void zero_tile(TileAcc<T>& acc, int cells) {
    uint4* w = reinterpret_cast<uint4*>(&acc);
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    for (int i = threadIdx.x; i < cells / 4; i += blockDim.x) {
        w[i] = z;
        if (sizeof(T) == 8) w[kTileX * kTileY / 4 + i] = z;
    }
}

// Writes the finished tile, two cells (int64) or four (uint32) per 16-byte
// store; rows of a tile start at even cells of a row of the mesh.
template <typename T>
__device__ __forceinline__ void store_tile(const TileAcc<T>& acc, bool split, const TileGeom& g,
                                           int c0, int r0, int cells, T* __restrict__ density) {
    const uint32_t* lo = reinterpret_cast<const uint32_t*>(&acc);
    if (sizeof(T) == 8) {
        const uint32_t* hi = lo + kTileX * kTileY;
        const int shift = split ? kSplitShift : 32;
        for (int i = 2 * threadIdx.x; i < cells; i += 2 * blockDim.x) {
            const uint2 l = *reinterpret_cast<const uint2*>(lo + i);
            const uint2 h = *reinterpret_cast<const uint2*>(hi + i);
            const int y = i >> g.tx_log2, x = i & (g.TX - 1);
            ulonglong2 v;
            v.x = ((unsigned long long)h.x << shift) + l.x;
            v.y = ((unsigned long long)h.y << shift) + l.y;
            *reinterpret_cast<ulonglong2*>(density + (size_t)(r0 + y) * g.MW + c0 + x) = v;
        }
    } else {
        for (int i = 4 * threadIdx.x; i < cells; i += 4 * blockDim.x) {
            const uint4 l = *reinterpret_cast<const uint4*>(lo + i);
            const int y = i >> g.tx_log2, x = i & (g.TX - 1);
            *reinterpret_cast<uint4*>(density + (size_t)(r0 + y) * g.MW + c0 + x) = l;
        }
    }
}

// One body's CIC corners, quantized, with their tile coordinates.
template <typename T>
struct Corners {
    int bx, by;     // CIC base, guarded (unwrapped)
    T q00, q10, q01, q11;
};

template <typename T>
__device__ __forceinline__ Corners<T> corners(float4 e, const TileGeom& g, float scale) {
    const float gx = __fsub_rn(__fmul_rn(e.x, (float)g.W), 0.5f);
    const float gy = __fsub_rn(__fmul_rn(e.y, (float)g.H), 0.5f);
    const float flx = floorf(gx), fly = floorf(gy);
    Corners<T> c;
    c.bx = guard_coord(float_to_int(flx), g.MW);
    c.by = guard_coord(float_to_int(fly), g.MH);
    const float fx = __fsub_rn(gx, flx), fy = __fsub_rn(gy, fly);
    const float ofx = __fsub_rn(1.0f, fx), ofy = __fsub_rn(1.0f, fy);
    const float m = e.z;
    c.q00 = quantize<T>(__fmul_rn(__fmul_rn(ofx, ofy), m), scale);
    c.q10 = quantize<T>(__fmul_rn(__fmul_rn(fx, ofy), m), scale);
    c.q01 = quantize<T>(__fmul_rn(__fmul_rn(ofx, fy), m), scale);
    c.q11 = quantize<T>(__fmul_rn(__fmul_rn(fx, fy), m), scale);
    return c;
}

template <typename T, bool SPLIT>
__device__ __forceinline__ void acc_put(TileAcc<T>& acc, int i, T v) {
    if (SPLIT) acc.add_split(i, v);
    else acc.add(i, v);
}

template <typename T>
__device__ __forceinline__ void add_node(TileAcc<T>& acc, const TileGeom& g, int c0, int r0,
                                         int nx, int ny, T v) {
    const int tx = wrap_index(nx, g.MW) - c0;
    const int ty = wrap_index(ny, g.MH) - r0;
    if ((unsigned)tx < (unsigned)g.TX && (unsigned)ty < (unsigned)g.TY) acc.add(ty * g.TX + tx, v);
}

template <typename T, bool SPLIT = false>
__device__ __forceinline__ void add_corners(const Corners<T>& c, const TileGeom& g, int c0, int r0,
                                            TileAcc<T>& acc) {
    const int x0 = wrap_index(c.bx, g.MW) - c0, x1 = wrap_index(c.bx + 1, g.MW) - c0;
    const int y0 = wrap_index(c.by, g.MH) - r0, y1 = wrap_index(c.by + 1, g.MH) - r0;
    const bool in_x0 = (unsigned)x0 < (unsigned)g.TX, in_x1 = (unsigned)x1 < (unsigned)g.TX;
    if ((unsigned)y0 < (unsigned)g.TY) {
        if (in_x0) acc_put<T, SPLIT>(acc, y0 * g.TX + x0, c.q00);
        if (in_x1) acc_put<T, SPLIT>(acc, y0 * g.TX + x1, c.q10);
    }
    if ((unsigned)y1 < (unsigned)g.TY) {
        if (in_x0) acc_put<T, SPLIT>(acc, y1 * g.TX + x0, c.q01);
        if (in_x1) acc_put<T, SPLIT>(acc, y1 * g.TX + x1, c.q11);
    }
}

// add_corners for a body whose CIC base lies in [0, MW-2] x [0, MH-2]: no
// mesh index wraps, so the tile coordinates are plain differences (the same
// cells wrap_index would give).
template <typename T, bool SPLIT>
__device__ __forceinline__ void add_corners_inner(const Corners<T>& c, const TileGeom& g, int c0,
                                                  int r0, TileAcc<T>& acc) {
    const int x0 = c.bx - c0, y0 = c.by - r0;
    const int i00 = y0 * g.TX + x0;
    const bool in_x0 = (unsigned)x0 < (unsigned)g.TX, in_x1 = (unsigned)(x0 + 1) < (unsigned)g.TX;
    const bool in_y0 = (unsigned)y0 < (unsigned)g.TY, in_y1 = (unsigned)(y0 + 1) < (unsigned)g.TY;
    if (in_y0 && in_x0) acc_put<T, SPLIT>(acc, i00, c.q00);
    if (in_y0 && in_x1) acc_put<T, SPLIT>(acc, i00 + 1, c.q10);
    if (in_y1 && in_x0) acc_put<T, SPLIT>(acc, i00 + g.TX, c.q01);
    if (in_y1 && in_x1) acc_put<T, SPLIT>(acc, i00 + g.TX + 1, c.q11);
}

// The split quantization of one corner weight w (int64 form, 2^-32 mass
// quanta): q = rint(w * 2^32) = floor(t) * 2^19 + rint(frac(t) * 2^19) with
// t = w * 2^13 (exact: a power-of-two scale), the first part an integer
// multiple of 2^19 so that rounding ties keep their parity. Both parts come
// out of float additions of 2^23, whose result's low bits are the integer:
// floor by a round-down addition, the fraction's rounding by the ordinary
// round-to-nearest-even one. Valid for t < 2^19 (q < 2^38); `large` records
// a larger weight. lo may be 2^19 itself.
__device__ __forceinline__ void split_quantize(float w, uint32_t& hi, uint32_t& lo, bool& large) {
    constexpr float kMagic = 8388608.0f;  // 2^23
    const float t = __fmul_rn(w, 8192.0f);
    const float a = __fadd_rd(t, kMagic);
    hi = __float_as_uint(a) - 0x4b000000u;
    const float rem = __fsub_rn(t, __fsub_rn(a, kMagic));
    lo = __float_as_uint(__fmaf_rn(rem, 524288.0f, kMagic)) - 0x4b000000u;
    large |= t >= 524288.0f;
}

// One body of a sparse tile whose CIC base lies inside the mesh with room
// for its +1 corner (0 <= gx < MW - 1, 0 <= gy < MH - 1, checked by the
// caller): floor by a round-down addition of 1.5 * 2^23 (|g| < 2^22), no
// wrap, the corner weights rounded like corners() (each product on its own,
// packed in pairs), then the four corners that land in the tile.
template <typename T>
__device__ __forceinline__ void fast_corners(float gx, float gy, float m, const TileGeom& g, int c0,
                                             int r0, float scale, TileAcc<T>& acc, bool& large) {
    constexpr float kFloorMagic = 12582912.0f;  // 1.5 * 2^23
    const float fxa = __fadd_rd(gx, kFloorMagic), fya = __fadd_rd(gy, kFloorMagic);
    const int bx = (int)(__float_as_uint(fxa) - 0x4b400000u);
    const int by = (int)(__float_as_uint(fya) - 0x4b400000u);
    const float fx = __fsub_rn(gx, __fsub_rn(fxa, kFloorMagic));
    const float fy = __fsub_rn(gy, __fsub_rn(fya, kFloorMagic));
    const float ofx = __fsub_rn(1.0f, fx), ofy = __fsub_rn(1.0f, fy);
    // (ofx*ofy, fx*ofy) and (ofx*fy, fx*fy), then each times m.
    const float2 r0w = __fmul2_rn(__fmul2_rn(make_float2(ofx, fx), make_float2(ofy, ofy)),
                                  make_float2(m, m));
    const float2 r1w = __fmul2_rn(__fmul2_rn(make_float2(ofx, fx), make_float2(fy, fy)),
                                  make_float2(m, m));
    const int x0 = bx - c0, y0 = by - r0;
    const int i00 = y0 * g.TX + x0;
    const bool in_x0 = (unsigned)x0 < (unsigned)g.TX, in_x1 = (unsigned)(x0 + 1) < (unsigned)g.TX;
    const bool in_y0 = (unsigned)y0 < (unsigned)g.TY, in_y1 = (unsigned)(y0 + 1) < (unsigned)g.TY;
    if (sizeof(T) == 8) {
        uint32_t h[4], l[4];
        split_quantize(r0w.x, h[0], l[0], large);
        split_quantize(r0w.y, h[1], l[1], large);
        split_quantize(r1w.x, h[2], l[2], large);
        split_quantize(r1w.y, h[3], l[3], large);
        uint32_t* lo = reinterpret_cast<uint32_t*>(&acc);
        uint32_t* hi = lo + kTileX * kTileY;
        if (in_y0 && in_x0) { atomicAdd(&lo[i00], l[0]); atomicAdd(&hi[i00], h[0]); }
        if (in_y0 && in_x1) { atomicAdd(&lo[i00 + 1], l[1]); atomicAdd(&hi[i00 + 1], h[1]); }
        if (in_y1 && in_x0) { atomicAdd(&lo[i00 + g.TX], l[2]); atomicAdd(&hi[i00 + g.TX], h[2]); }
        if (in_y1 && in_x1) {
            atomicAdd(&lo[i00 + g.TX + 1], l[3]);
            atomicAdd(&hi[i00 + g.TX + 1], h[3]);
        }
    } else {
        uint32_t* lo = reinterpret_cast<uint32_t*>(&acc);
        if (in_y0 && in_x0) atomicAdd(&lo[i00], __float2uint_rn(__fmul_rn(r0w.x, scale)));
        if (in_y0 && in_x1) atomicAdd(&lo[i00 + 1], __float2uint_rn(__fmul_rn(r0w.y, scale)));
        if (in_y1 && in_x0) atomicAdd(&lo[i00 + g.TX], __float2uint_rn(__fmul_rn(r1w.x, scale)));
        if (in_y1 && in_x1)
            atomicAdd(&lo[i00 + g.TX + 1], __float2uint_rn(__fmul_rn(r1w.y, scale)));
    }
}

// Sparse tiles: warp w takes the w-th share of the runs' positions, its
// lanes consecutive positions (coalesced within a run), four loads in flight
// per lane; each lane walks the runs forward from one search, so finding an
// entry costs O(1). Each body's corners are added one by one, without index
// wrapping where none can occur. SPLIT: the split accumulator form; returns
// (in every thread) whether a value was too large for it.
template <typename T, bool SPLIT>
__device__ bool tile_direct(const float4* __restrict__ entries, int total, const int* run_begin,
                            const int* run_prefix, const TileGeom& g, int c0, int r0, float scale,
                            TileAcc<T>& acc) {
    bool large = false;
    constexpr int U = 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const int share = (total + warps - 1) / warps;
    const int kb = min(total, warp * share), ke = min(total, kb + share);
    int r = 0;
    {
        int lo = 0, hi = kMaxRuns - 1;
        const int k = kb + lane;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (run_prefix[mid] <= k) lo = mid;
            else hi = mid - 1;
        }
        r = lo;
    }
    for (int p0 = kb + lane; p0 < ke; p0 += 32 * U) {
        float4 e[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int p = p0 + 32 * u;
            if (p < ke) {
                while (r + 1 < kMaxRuns && run_prefix[r + 1] <= p) ++r;
                e[u] = __ldg(&entries[run_begin[r] + (p - run_prefix[r])]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (p0 + 32 * u >= ke) continue;
            if (SPLIT) {
                const float gx = __fsub_rn(__fmul_rn(e[u].x, (float)g.W), 0.5f);
                const float gy = __fsub_rn(__fmul_rn(e[u].y, (float)g.H), 0.5f);
                if (gx >= 0.0f && gx < (float)(g.MW - 1) && gy >= 0.0f && gy < (float)(g.MH - 1)) {
                    fast_corners<T>(gx, gy, e[u].z, g, c0, r0, scale, acc, large);
                    continue;
                }
            }
            const Corners<T> c = corners<T>(e[u], g, scale);
            if (SPLIT)
                large |= TileAcc<T>::too_large(c.q00) | TileAcc<T>::too_large(c.q10) |
                         TileAcc<T>::too_large(c.q01) | TileAcc<T>::too_large(c.q11);
            if ((unsigned)c.bx <= (unsigned)(g.MW - 2) && (unsigned)c.by <= (unsigned)(g.MH - 2))
                add_corners_inner<T, SPLIT>(c, g, c0, r0, acc);
            else
                add_corners<T, SPLIT>(c, g, c0, r0, acc);
        }
    }
    return __syncthreads_or(large ? 1 : 0) != 0;
}

// Sums of consecutive bodies of one home cell (hx, hy) over the 3x3 mesh
// nodes around it: a body deposits into the 2x2 of them that start at its
// CIC base (hx-1 or hx, hy-1 or hy).
template <typename T>
struct CellSums {
    int hx, hy;  // unwrapped home column / row; hx == INT_MIN: none open
    T a[9];
};

template <typename T>
__device__ __forceinline__ void flush_cell(CellSums<T>& s, TileAcc<T>& acc, const TileGeom& g,
                                           int c0, int r0) {
    if (s.hx == INT_MIN) return;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        if (s.a[q] != T(0)) add_node<T>(acc, g, c0, r0, s.hx - 1 + q % 3, s.hy - 1 + q / 3, s.a[q]);
        s.a[q] = T(0);
    }
}

// Dense tiles: thread t takes the t-th share of positions [kb, ke) of the
// runs (contiguous, so consecutive bodies mostly share a home cell) and
// sums them per cell in registers; the cells still open at the end are
// merged across the warp (equal cells sit in consecutive lanes: the runs
// are in cell order) before touching the tile. A dense cell thus costs one
// shared atomic per node and warp, not per body. Every thread of the block
// calls this.
template <typename T>
__device__ void tile_dense(const float4* __restrict__ entries, int kb, int ke, const int* run_begin,
                           const int* run_end, const int* run_prefix, const TileGeom& g, int c0,
                           int r0, float scale, TileAcc<T>& acc) {
    const int lane = threadIdx.x & 31;
    const int len = ke - kb, per = (len + (int)blockDim.x - 1) / (int)blockDim.x;
    int k = kb + min(len, (int)threadIdx.x * per);
    const int k1 = kb + min(len, (int)threadIdx.x * per + per);
    CellSums<T> s;
    s.hx = INT_MIN;
    s.hy = 0;
#pragma unroll
    for (int q = 0; q < 9; ++q) s.a[q] = T(0);
    if (k < k1) {
        int r = 0;
        {
            int lo = 0, hi = kMaxRuns - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (run_prefix[mid] <= k) lo = mid;
                else hi = mid - 1;
            }
            r = lo;
        }
        int idx = run_begin[r] + (k - run_prefix[r]);
        float4 next = __ldg(&entries[idx]);
        for (; k < k1; ++k) {
            const float4 en = next;
            // Advance to the following entry (next run when this one ends)
            // and start its load before working on this one.
            ++idx;
            if (k + 1 < k1) {
                while (idx >= run_end[r] && r + 1 < kMaxRuns) { ++r; idx = run_begin[r]; }
                next = __ldg(&entries[idx]);
            }
            const Corners<T> c = corners<T>(en, g, scale);
            const int hx = float_to_int(floorf(__fmul_rn(en.x, (float)g.W)));
            const int hy = float_to_int(floorf(__fmul_rn(en.y, (float)g.H)));
            const int ox = c.bx - hx, oy = c.by - hy;
            if ((ox != -1 && ox != 0) || (oy != -1 && oy != 0)) {
                add_corners<T>(c, g, c0, r0, acc);  // a position outside the domain
                continue;
            }
            if (hx != s.hx || hy != s.hy) {
                flush_cell<T>(s, acc, g, c0, r0);
                s.hx = hx;
                s.hy = hy;
            }
            const int base = (oy + 1) * 3 + (ox + 1);  // node of corner (0, 0): 0, 1, 3 or 4
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const int d = q - base;
                s.a[q] += d == 0 ? c.q00 : d == 1 ? c.q10 : d == 3 ? c.q01 : d == 4 ? c.q11 : T(0);
            }
        }
    }
    const long long key = s.hx == INT_MIN
                              ? LLONG_MIN
                              : (long long)(((unsigned long long)(unsigned)s.hy << 32) | (unsigned)s.hx);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long ok = __shfl_up_sync(0xffffffffu, key, o);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const T v = __shfl_up_sync(0xffffffffu, s.a[q], o);
            if (lane >= o && ok == key) s.a[q] += v;
        }
    }
    const long long nk = __shfl_down_sync(0xffffffffu, key, 1);
    if (lane == 31 || nk != key) flush_cell<T>(s, acc, g, c0, r0);
}

// Average bodies per tile cell above which a tile is summed per cell.
constexpr int kDenseBodiesPerCell = 2;

template <typename T>
__global__ void __launch_bounds__(kThreads) deposit_tiles_kernel(
    const float4* __restrict__ entries, const int* __restrict__ cell_start, TileGeom g,
    float scale, T* __restrict__ density, int4* __restrict__ work, int* __restrict__ work_count,
    int work_capacity) {
    grid_dependency_wait();
    __shared__ __align__(16) TileAcc<T> acc;
    __shared__ int run_begin[kMaxRuns], run_end[kMaxRuns], run_prefix[kMaxRuns];
    __shared__ int s_total;
    const int tile = blockIdx.x;
    const int c0 = (tile % g.tiles_x) * g.TX, r0 = (tile / g.tiles_x) * g.TY;
    const int cells = g.TX * g.TY;
    zero_tile<T>(acc, cells);
    const int total = tile_runs(cell_start, g, tile, run_begin, run_end, run_prefix, &s_total);
    bool split = false;  // uniform over the CTA
    if (total > kTileCap) {
        // Heavy tile: zeros now; its runs, in pieces of kPiece entries, to
        // the second kernel.
        if (threadIdx.x == 0) {
            const int pieces = (total + kPiece - 1) / kPiece;
            const int base = atomicAdd(work_count, pieces);
            for (int j = 0; j < pieces && base + j < work_capacity; ++j)
                work[base + j] = make_int4(tile, j * kPiece, min(total, (j + 1) * kPiece), 0);
        }
    } else if (total >= kDenseBodiesPerCell * cells) {
        tile_dense<T>(entries, 0, total, run_begin, run_end, run_prefix, g, c0, r0, scale, acc);
    } else {
        split = true;
        if (tile_direct<T, true>(entries, total, run_begin, run_prefix, g, c0, r0, scale, acc)) {
            // A body of mass 64 or more: the same tile again, carrying.
            split = false;
            zero_tile<T>(acc, cells);
            __syncthreads();
            tile_direct<T, false>(entries, total, run_begin, run_prefix, g, c0, r0, scale, acc);
        }
    }
    __syncthreads();
    store_tile<T>(acc, split, g, c0, r0, cells, density);
}

// Pieces of heavy tiles: each warp takes a 1/warps share of the piece
// (summed per cell), then the tile's non-zero sums go to global atomics.
template <typename T>
__global__ void __launch_bounds__(kThreads) deposit_heavy_kernel(
    const float4* __restrict__ entries, const int* __restrict__ cell_start, TileGeom g,
    float scale, T* __restrict__ density, const int4* __restrict__ work,
    const int* __restrict__ work_count, int work_capacity) {
    grid_dependency_wait();
    __shared__ TileAcc<T> acc;
    __shared__ int run_begin[kMaxRuns], run_end[kMaxRuns], run_prefix[kMaxRuns];
    __shared__ int s_total;
    const int items = min(*work_count, work_capacity);
    const int cells = g.TX * g.TY;
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int4 w = work[item];
        const int tile = w.x;
        const int c0 = (tile % g.tiles_x) * g.TX, r0 = (tile / g.tiles_x) * g.TY;
        for (int i = threadIdx.x; i < cells; i += blockDim.x) acc.zero(i);
        tile_runs(cell_start, g, tile, run_begin, run_end, run_prefix, &s_total);
        tile_dense<T>(entries, w.y, w.z, run_begin, run_end, run_prefix, g, c0, r0, scale, acc);
        __syncthreads();
        for (int i = threadIdx.x; i < cells; i += blockDim.x) {
            const T v = acc.get(i);
            const int y = i >> g.tx_log2, x = i & (g.TX - 1);
            if (v != T(0)) atomicAdd(&density[(size_t)(r0 + y) * g.MW + c0 + x], v);
        }
        __syncthreads();  // acc is reused by the next item
    }
}

// Small and clustered workloads: one CTA per kChunkEntries consecutive
// entries of the cell order (perfect balance whatever the clustering). Their
// CIC footprint lies in the row-major mesh window [(y0-1)*MW + x0-1,
// (y1+1)*MW + x1+1]; the CTA accumulates it in shared memory and flushes each
// non-zero cell with one global atomic into the cleared mesh. Deposits that
// wrap across the mesh edge, or that fall beyond the window's capacity, go
// straight to global memory.
constexpr int kChunkEntries = 1024;
constexpr int kWindowBytes = 48 * 1024;

template <typename T>
__device__ __forceinline__ void deposit_chunks_body(
    int block, const float4* __restrict__ entries, const uint32_t* __restrict__ keys, int n, int W,
    int H, int MW, int MH, float scale, T* __restrict__ density, int window_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* window = reinterpret_cast<T*>(smem_raw);
    __shared__ long long s_lo;
    __shared__ int s_len;

    const int base = block * kChunkEntries;
    const int count = min(kChunkEntries, n - base);
    if (threadIdx.x == 0) {
        const uint32_t c0 = keys[base], c1 = keys[base + count - 1];
        const int x0 = (int)(c0 % (uint32_t)W), y0 = (int)(c0 / (uint32_t)W);
        const int x1 = (int)(c1 % (uint32_t)W), y1 = (int)(c1 / (uint32_t)W);
        long long lo = (long long)(y0 - 1) * MW + (x0 - 1);
        long long hi = (long long)(y1 + 1) * MW + (x1 + 1);
        if (lo < 0) lo = 0;
        long long len = hi - lo + 1;
        if (len > window_cap) len = window_cap;
        s_lo = lo;
        s_len = (int)len;
    }
    __syncthreads();
    const long long lo = s_lo;
    const int len = s_len;
    for (int i = threadIdx.x; i < len; i += blockDim.x) window[i] = T(0);
    __syncthreads();

    for (int k = threadIdx.x; k < count; k += blockDim.x) {
        const float4 e = entries[base + k];
        const float gx = __fsub_rn(__fmul_rn(e.x, (float)W), 0.5f);
        const float gy = __fsub_rn(__fmul_rn(e.y, (float)H), 0.5f);
        const float flx = floorf(gx), fly = floorf(gy);
        const int bx = guard_coord(float_to_int(flx), MW), by = guard_coord(float_to_int(fly), MH);
        const float fx = __fsub_rn(gx, flx), fy = __fsub_rn(gy, fly);
        const float ofx = __fsub_rn(1.0f, fx), ofy = __fsub_rn(1.0f, fy);
        const float m = e.z;
        float w[4];
        w[0] = __fmul_rn(__fmul_rn(ofx, ofy), m);
        w[1] = __fmul_rn(__fmul_rn(fx, ofy), m);
        w[2] = __fmul_rn(__fmul_rn(ofx, fy), m);
        w[3] = __fmul_rn(__fmul_rn(fx, fy), m);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int mx = wrap_index(bx + (q & 1), MW), my = wrap_index(by + (q >> 1), MH);
            const long long idx = (long long)mx + (long long)my * MW;
            const T v = quantize<T>(w[q], scale);
            const long long off = idx - lo;
            if (off >= 0 && off < len) atomicAdd(&window[off], v);
            else atomicAdd(&density[idx], v);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
        const T v = window[i];
        if (v != T(0)) atomicAdd(&density[lo + i], v);
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) deposit_chunks_kernel(
    const float4* __restrict__ entries, const uint32_t* __restrict__ keys, int n, int W, int H,
    int MW, int MH, float scale, T* __restrict__ density, int window_cap) {
    grid_dependency_wait();
    deposit_chunks_body<T>(blockIdx.x, entries, keys, n, W, H, MW, MH, scale, density, window_cap);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) deposit_chunks_batched_kernel(
    const DepositArgs* __restrict__ args, const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const DepositArgs a = args[sb.x];
    deposit_chunks_body<T>(sb.y, a.entries, a.keys, a.n, a.W, a.H, a.MW, a.MH, a.scale,
                           static_cast<T*>(a.density), kWindowBytes / (int)sizeof(T));
}

TileGeom tile_geom(const GridShape& g) {
    TileGeom t;
    t.W = g.W; t.H = g.H; t.MW = g.MW; t.MH = g.MH;
    t.TX = g.MW < kTileX ? g.MW : kTileX;
    t.TY = g.MH < kTileY ? g.MH : kTileY;
    t.tiles_x = g.MW / t.TX;
    t.tx_log2 = 0;
    while ((1 << t.tx_log2) < t.TX) ++t.tx_log2;
    return t;
}

}  // namespace

// Host-side launchers: not part of the coherent copy of the bodies that the
// batched form's persistent kernel uses (p3m_step.cu).
#ifndef P3M_COHERENT_BODIES

cudaError_t configure_deposit() {
    const void* fns[] = {(const void*)deposit_chunks_kernel<unsigned long long>,
                         (const void*)deposit_chunks_kernel<uint32_t>,
                         (const void*)deposit_chunks_batched_kernel<unsigned long long>,
                         (const void*)deposit_chunks_batched_kernel<uint32_t>};
    for (const void* f : fns) {
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kWindowBytes);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int chunk_deposit_blocks(int n) { return n > 0 ? (n + kChunkEntries - 1) / kChunkEntries : 0; }
int chunk_deposit_smem() { return kWindowBytes; }

cudaError_t batched_deposit(const DepositArgs* a, BatchGrid g, int deposit_mode, cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    if (deposit_mode == P3M_DEPOSIT_I64)
        deposit_chunks_batched_kernel<unsigned long long><<<g.blocks, kThreads, kWindowBytes, s>>>(
            a, g.first, g.sims);
    else
        deposit_chunks_batched_kernel<uint32_t><<<g.blocks, kThreads, kWindowBytes, s>>>(
            a, g.first, g.sims);
    count_launches(1);
    return cudaGetLastError();
}

bool deposit_uses_cell_starts(int n) { return n >= kTileMinBodies; }

size_t deposit_work_entries(int capacity, int MW, int MH) {
    // Each body lies in the runs of at most 2 x 2 tiles; a tile has at most
    // kMaxRuns runs, each cut into pieces of kPiece.
    const int tx = MW < kTileX ? MW : kTileX, ty = MH < kTileY ? MH : kTileY;
    const size_t tiles = (size_t)(MW / tx) * (size_t)(MH / ty);
    return 4 * ((size_t)capacity / kPiece + 1) + tiles;
}

cudaError_t launch_deposit(const float4* entries, const uint32_t* keys, const int* cell_start,
                           int n, GridShape g, int deposit_mode, float mass_scale, void* density,
                           int4* work, int* work_count, int work_capacity, cudaStream_t stream) {
    const bool i64 = deposit_mode == P3M_DEPOSIT_I64;
    if (n < kTileMinBodies) {
        cudaError_t e = cudaMemsetAsync(density, 0, (size_t)g.MW * g.MH * (i64 ? 8 : 4), stream);
        if (e != cudaSuccess || n <= 0) return e;
        const int blocks = (n + kChunkEntries - 1) / kChunkEntries;
        if (i64) {
            using T = unsigned long long;
            launch_chained(deposit_chunks_kernel<T>, blocks, kThreads, kWindowBytes, stream,
                entries, keys, n, g.W, g.H, g.MW, g.MH, 4294967296.0f, static_cast<T*>(density),
                kWindowBytes / (int)sizeof(T));
        } else {
            using T = uint32_t;
            launch_chained(deposit_chunks_kernel<T>, blocks, kThreads, kWindowBytes, stream,
                entries, keys, n, g.W, g.H, g.MW, g.MH, mass_scale, static_cast<T*>(density),
                kWindowBytes / (int)sizeof(T));
        }
        count_launches(1);
        return cudaGetLastError();
    }
    const TileGeom t = tile_geom(g);
    const int tiles = t.tiles_x * (g.MH / t.TY);
    cudaError_t e = cudaMemsetAsync(work_count, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    int heavy_blocks = 4 * 148;
    if (heavy_blocks > work_capacity) heavy_blocks = work_capacity > 0 ? work_capacity : 1;
    if (deposit_mode == P3M_DEPOSIT_I64) {
        using T = unsigned long long;
        launch_chained(deposit_tiles_kernel<T>, tiles, kThreads, 0, stream,
            entries, cell_start, t, 4294967296.0f, static_cast<T*>(density), work, work_count,
            work_capacity);
        launch_chained(deposit_heavy_kernel<T>, heavy_blocks, kThreads, 0, stream,
            entries, cell_start, t, 4294967296.0f, static_cast<T*>(density), work, work_count,
            work_capacity);
    } else {
        using T = uint32_t;
        launch_chained(deposit_tiles_kernel<T>, tiles, kThreads, 0, stream,
            entries, cell_start, t, mass_scale, static_cast<T*>(density), work, work_count,
            work_capacity);
        launch_chained(deposit_heavy_kernel<T>, heavy_blocks, kThreads, 0, stream,
            entries, cell_start, t, mass_scale, static_cast<T*>(density), work, work_count,
            work_capacity);
    }
    count_launches(2);
    return cudaGetLastError();
}

#endif  // !P3M_COHERENT_BODIES
}  // namespace p3m
