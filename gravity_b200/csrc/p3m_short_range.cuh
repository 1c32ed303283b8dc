// p3m_short_range.cuh — the short-range correction kernel (kick.comp:122-151).
//
// The short-range complement of the Gaussian split, summed over the
// (2Rx+1)x(2Ry+1) cell stencil around each body's home cell: cells holding
// more than `exact` bodies act as a monopole at the cell centre with the
// fixed-point cell mass; other cells, and the home cell up to `home_limit`
// list entries, are summed body by body in list order (descending ID), the
// body itself skipped. The result goes to a_short[id]; the interpolation +
// kick kernel adds it.
//
// One thread per body in ID order: after the Morton reorder IDs follow screen
// tiles, so a warp's stencils overlap in 2D and the cell tables and
// neighbour entries come from L1/L2. The stencil radii are template
// parameters and the loops are unrolled; the wrapped column/row of every
// stencil offset and its periodic image shift are computed once per target.
//
// EXACT = 2 (the reference's default exactNeighborBodyLimit) runs every
// non-home stencil cell without branches: two source slots per cell, filled
// by predicated loads of the cell's first two list entries, or the monopole
// and an empty slot; a missing source has mass 0 and adds exactly 0, so every
// lane of a warp does the same work whatever its cells hold. EXACT = 0 walks
// the lists for any other limit.
//
// The pair term G m exp(-r^2/2s^2) d / (M max(r^2, r_min^2)) is evaluated as
// (G/M) m exp2(-r^2 log2(e)/2s^2) * rcp(max(r^2, r_min^2)) * d with fused
// multiply-adds. On the torus the reference takes the minimum image
// (kick.comp:68); every stencil here spans at most 13 cells of a grid of at
// least 16, so the image of a neighbour cell is fixed by how its column and
// row wrapped, and the source position is shifted by that image instead of
// rounding the displacement. Forces agree with the oracle's literal FP32
// evaluation to ~1e-7 relative per term (another summation order and
// rounding); the contract is 1e-5 relative RMS.
//
// Each p3m_short_range_rN.cu instantiates one Rx so the instantiations
// compile in parallel.
// Included once as it is, and once more by p3m_step.cu inside namespace
// p3m::coherent (P3M_COHERENT_BODIES) for the batched form's persistent
// kernel, which must not read through the non-coherent load path.
#if defined(P3M_COHERENT_BODIES) ? !defined(P3M_SHORT_RANGE_COHERENT_) : !defined(P3M_SHORT_RANGE_PLAIN_)
#ifdef P3M_COHERENT_BODIES
#define P3M_SHORT_RANGE_COHERENT_
#else
#define P3M_SHORT_RANGE_PLAIN_
#endif

#include "p3m_internal.cuh"

namespace p3m {
namespace sr {

struct PairConst {
    float aspect;
    float neg_log2e_over_2s2;  // -log2(e) / (2 sigma^2)
    float min_dist2;           // (min_frac * min(cell w, cell h))^2
    float g_over_m;            // G / M_tot
};

__device__ __forceinline__ PairConst pair_const(const KickParams& p) {
    PairConst k;
    k.aspect = p.aspect;
    const float sigma = p.sigma_cells / (float)p.H;
    k.neg_log2e_over_2s2 = -1.4426950408889634f / (2.0f * sigma * sigma);
    const float cw = p.aspect / (float)p.W, ch = 1.0f / (float)p.H;
    const float md = p.min_frac * fminf(cw, ch);
    k.min_dist2 = md * md;
    k.g_over_m = p.gravity / p.total_mass;
    return k;
}

// 2^x by the hardware's approximate exponential (relative error below
// 2^-22; denormal results flush to zero — the weight here is at least
// exp(-r^2 / 2 sigma^2) over a 13-cell stencil, far above that range).
__device__ __forceinline__ float fast_exp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// (dx, dy): source minus target in unit coordinates, already on the right
// image. Adds G m exp(-r^2/2s^2) d / (M max(r^2, r_min^2)).
__device__ __forceinline__ void pair_add(const PairConst& k, float dx, float dy, float m,
                                         float& ax, float& ay) {
    const float px = dx * k.aspect;
    const float r2 = fmaf(px, px, dy * dy);
    const float w = fast_exp2(r2 * k.neg_log2e_over_2s2);
    const float phys = __fdividef(k.g_over_m * m * w, fmaxf(r2, k.min_dist2));
    ax = fmaf(phys, dx, ax);  // (phys * px) / aspect == phys * dx
    ay = fmaf(phys, dy, ay);
}

// 1/x by the hardware's approximate reciprocal (PTX rcp.approx.ftz.f32): the
// pair term's division is by max(r^2, r_min^2), far from the flushed range.
__device__ __forceinline__ float fast_rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Two sources at once with Blackwell's packed FP32x2 arithmetic (each half
// rounded as one scalar operation): the pair term of pair_add with the
// source's G m / M_tot already formed (`gm`), source 0 in .x and source 1 in
// .y, accumulated into (ax, ay) per half.
__device__ __forceinline__ void pair_add2_gm(const PairConst& k, float2 dx, float2 dy, float2 gm,
                                             float2& ax, float2& ay) {
    const float2 px = __fmul2_rn(dx, make_float2(k.aspect, k.aspect));
    const float2 r2 = __ffma2_rn(px, px, __fmul2_rn(dy, dy));
    const float2 e = __fmul2_rn(r2, make_float2(k.neg_log2e_over_2s2, k.neg_log2e_over_2s2));
    const float2 num = __fmul2_rn(gm, make_float2(fast_exp2(e.x), fast_exp2(e.y)));
    const float2 inv = make_float2(fast_rcp(fmaxf(r2.x, k.min_dist2)),
                                   fast_rcp(fmaxf(r2.y, k.min_dist2)));
    const float2 phys = __fmul2_rn(num, inv);
    ax = __ffma2_rn(phys, dx, ax);
    ay = __ffma2_rn(phys, dy, ay);
}

// Cells of the slot table a CTA stages in shared memory (24 bytes each): the
// box spanned by its bodies' stencils, when it holds at most this many.
constexpr int kStageCells = 1536;

struct StageBox {
    int x0, y0, w, h;  // box origin (unwrapped cell coordinates), width, height
    bool staged;
};

// The two-slot form (EXACT = 2) stages, per CTA, the slot-table box covering
// every stencil of its bodies: after the Morton reorder a CTA's bodies are a
// compact patch, so the box is a few hundred cells that every lane then reads
// from shared memory instead of each lane fetching its 48 cells through L1.
// A CTA whose box is larger than kStageCells (a patch split across the torus
// seam, or sparse bodies) reads the table from global memory. All threads of
// the CTA take part (none may have returned). stage_box finds the box (one
// barrier); stage_fill loads it (another barrier), so a caller can issue
// loads of its own between the two.
template <int RX, int RY>
__device__ __forceinline__ StageBox stage_box(bool valid, int hx, int hy, int* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const int mnx = __reduce_min_sync(0xffffffffu, valid ? hx : 0x7fffffff);
    const int mxx = __reduce_max_sync(0xffffffffu, valid ? hx : (int)0x80000000);
    const int mny = __reduce_min_sync(0xffffffffu, valid ? hy : 0x7fffffff);
    const int mxy = __reduce_max_sync(0xffffffffu, valid ? hy : (int)0x80000000);
    if (lane == 0) {
        red[warp * 4 + 0] = mnx;
        red[warp * 4 + 1] = mxx;
        red[warp * 4 + 2] = mny;
        red[warp * 4 + 3] = mxy;
    }
    __syncthreads();
    int x0 = 0x7fffffff, x1 = (int)0x80000000, y0 = 0x7fffffff, y1 = (int)0x80000000;
    for (int w = 0; w < warps; ++w) {
        x0 = min(x0, red[w * 4 + 0]);
        x1 = max(x1, red[w * 4 + 1]);
        y0 = min(y0, red[w * 4 + 2]);
        y1 = max(y1, red[w * 4 + 3]);
    }
    StageBox box;
    box.x0 = x0 - RX;
    box.y0 = y0 - RY;
    const long long bw = (long long)x1 - x0 + 1 + 2 * RX;
    const long long bh = (long long)y1 - y0 + 1 + 2 * RY;
    box.w = (int)bw;
    box.staged = bw * bh <= kStageCells;
    box.h = box.staged ? (int)bh : 0;
    return box;
}

__device__ __forceinline__ void stage_fill(const StageBox& box, const float4* __restrict__ slots,
                                           const float2* __restrict__ slots_b,
                                           const KickParams& p, float4* st_a, float2* st_b) {
    if (box.staged) {
        const int cells = box.w * box.h;
        // Row of box cell c: floor((c + 0.5) / w) in FP32 instead of an
        // integer division. (c + 0.5) / w lies at least 0.5 / w from an
        // integer, and for c < kStageCells the two roundings move it by less
        // than 2e-4 / w, so the floor is exact (checked for every w and c).
        const float inv_w = 1.0f / (float)box.w;
        // Two cells per thread per round: 512 at 256 threads, a typical box
        // (about 22 x 22) in one round, with registers left for the home
        // cell's entries in flight meanwhile.
        constexpr int kBatch = 2;
        for (int c0 = threadIdx.x; c0 < cells; c0 += kBatch * blockDim.x) {
            float4 va[kBatch];
            float2 vb[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int c = c0 + u * blockDim.x;
                va[u] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                vb[u] = make_float2(0.0f, 0.0f);
                if (c < cells) {
                    const int r = (int)(((float)c + 0.5f) * inv_w);
                    const int cx = box.x0 + (c - r * box.w), cy = box.y0 + r;
                    // Cells beyond a wall are never read: their slots stay
                    // massless zeros.
                    if (!p.bounded || (cx >= 0 && cx < p.W && cy >= 0 && cy < p.H)) {
                        const int wx = wrap_index(cx, p.W), wy = wrap_index(cy, p.H);
                        const int cell = wy * p.W + wx;
                        va[u] = __ldg(&slots[cell]);
                        vb[u] = __ldg(&slots_b[cell]);
                        // The slots moved to the box's image of the cell, as
                        // the global-table path shifts them per stencil cell.
                        const float sx = (float)(cx - wx) * (1.0f / (float)p.W);
                        const float sy = (float)(cy - wy) * (1.0f / (float)p.H);
                        va[u] = make_float4(va[u].x + sx, va[u].y + sx, va[u].z + sy,
                                            va[u].w + sy);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int c = c0 + u * blockDim.x;
                if (c < cells) {
                    st_a[c] = va[u];
                    st_b[c] = vb[u];
                }
            }
        }
    }
    __syncthreads();
}

// One step of a list walk: entries o0 and o1 (o1 present when has1) of a
// cell whose image shift is (sx, sy), against the target at -(ntx, nty). The
// target itself and the filler of an odd count have mass 0 and add nothing.
__device__ __forceinline__ void walk_step(const PairConst& k, float4 o0, float4 o1, bool has1,
                                          uint32_t id, float2 sx, float2 sy, float2 ntx,
                                          float2 nty, float2& ax2, float2& ay2) {
    const float m0 = __float_as_uint(o0.w) != id ? o0.z : 0.0f;
    const float m1 = has1 && __float_as_uint(o1.w) != id ? o1.z : 0.0f;
    // (o + shift) - t, rounded as the scalar form does.
    const float2 dx = __fadd2_rn(__fadd2_rn(make_float2(o0.x, o1.x), sx), ntx);
    const float2 dy = __fadd2_rn(__fadd2_rn(make_float2(o0.y, o1.y), sy), nty);
    pair_add2_gm(k, dx, dy,
                 __fmul2_rn(make_float2(k.g_over_m, k.g_over_m), make_float2(m0, m1)), ax2,
                 ay2);
}

// The home cell of the two-slot form, read before the stencil: its list walk
// (min(count, home_limit) entries from `start`) and the first two entries,
// loaded while the CTA stages its slots.
struct HomeCell {
    int walk, start;
    float4 e0, e1;
};

// The stencil sum of one target (its position t, ID id, home cell hx, hy),
// accumulated per packed half: the two slots of a non-home cell (EXACT = 2),
// two list entries at a time in a walked cell, and a monopole in .x.
// STAGED: the slots come from the CTA's shared-memory box (base `sbase`, row
// pitch `bw`), else from the global table. The two instantiations keep the
// CTA-uniform choice out of the unrolled 49-cell loop. The two-slot form sums
// the home cell (`home_cell`) first, then the other cells row by row; the list
// form takes every cell, the home cell included, row by row.
template <int RX, int RY, int EXACT, bool STAGED>
__device__ __forceinline__ void stencil_sum(
    float4 t, uint32_t id, int hx, int hy, const PairConst& k, const KickParams& p,
    const float4* __restrict__ entries, const int* __restrict__ cell_start,
    const int* __restrict__ cell_count, const uint32_t* __restrict__ cell_mass,
    const float4* __restrict__ slots, const float2* __restrict__ slots_b, const float4* st_a,
    const float2* st_b, int sbase, int bw, const HomeCell& home_cell, float2& acc_x,
    float2& acc_y) {
    const float inv_w = 1.0f / (float)p.W, inv_h = 1.0f / (float)p.H;
    // Per stencil column: wrapped column, periodic image shift, validity. A
    // source at x on a column is at dx = (x + shift) - t.x, rounded twice as
    // written (exactly x - t.x where the column did not wrap). The staged
    // slots carry their shift already, so the staged two-slot loop needs
    // none of these per column.
    int col[2 * RX + 1];
    float shift_x[2 * RX + 1];
    bool ok_x[2 * RX + 1];
#pragma unroll
    for (int a = 0; a < 2 * RX + 1; ++a) {
        const int cx = hx + a - RX;
        const int wx = wrap_index(cx, p.W);
        col[a] = wx;
        shift_x[a] = (float)(cx - wx) * inv_w;
        ok_x[a] = !p.bounded || (cx >= 0 && cx < p.W);
    }
    const float2 neg_t = make_float2(-t.x, -t.y);
    const float2 ntx = make_float2(neg_t.x, neg_t.x), nty = make_float2(neg_t.y, neg_t.y);
    float2 ax2 = make_float2(0.0f, 0.0f), ay2 = make_float2(0.0f, 0.0f);
    if (EXACT == 2 && home_cell.walk > 0) {
        // The home cell never wraps: no image shift.
        const float2 zero = make_float2(0.0f, 0.0f);
        walk_step(k, home_cell.e0, home_cell.e1, home_cell.walk > 1, id, zero, zero, ntx, nty,
                  ax2, ay2);
        for (int e = 2; e < home_cell.walk; e += 2) {
            const float4 o0 = __ldg(&entries[home_cell.start + e]);
            const bool has1 = e + 1 < home_cell.walk;
            const float4 o1 = has1 ? __ldg(&entries[home_cell.start + e + 1]) : o0;
            walk_step(k, o0, o1, has1, id, zero, zero, ntx, nty, ax2, ay2);
        }
    }
    // The two-slot form unrolls the whole stencil (straight-line slot loads
    // and pair terms); the list walk keeps its rows rolled: unrolled, its
    // 49 branching cell walks outgrew the instruction cache (instruction-
    // fetch stalls dominated its ncu profile). Both kernels are held to 64
    // registers (4 CTAs per SM), which the rolled walk needs: without the
    // bound it took 94 in the batched kernel and lost a third of the warps.
    constexpr int kRowUnroll = EXACT == 2 ? 2 * RY + 1 : 1;
    // The staged two-slot loop takes every stencil cell: the stage holds
    // massless slots beyond a wall, whose terms are exact zeros (G m = 0
    // times a finite weight), and adding a zero leaves the accumulators'
    // bits as they are (they start at +0 and never become -0), the same
    // bits as skipping the cell as the other paths do.
    constexpr bool kWallChecks = !(EXACT == 2 && STAGED);
#pragma unroll kRowUnroll
    for (int b = 0; b < 2 * RY + 1; ++b) {
        const int cy = hy + b - RY;
        if (kWallChecks && p.bounded && (cy < 0 || cy >= p.H)) continue;
        const int wy = wrap_index(cy, p.H);
        const int row = wy * p.W;
        const float shift_y = (float)(cy - wy) * inv_h;
        const float cyr = ((float)wy + 0.5f) * inv_h;  // wrapped row centre
#pragma unroll
        for (int a = 0; a < 2 * RX + 1; ++a) {
            if (kWallChecks && !ok_x[a]) continue;
            const int index = row + col[a];
            const bool home = (a == RX) && (b == RY);
            if (EXACT == 2 && home) continue;  // summed first
            if (EXACT == 2) {
                // The cell's two slots, prepared once per step (cell_slots):
                // (x0, x1, y0, y1) and (G m0 / M_tot, G m1 / M_tot), so each
                // packed operand is one loaded register pair.
                float4 s0;
                float2 s1, dx, dy;
                if (STAGED) {
                    const int si = sbase + b * bw + a;
                    s0 = st_a[si];
                    s1 = st_b[si];
                    dx = __fadd2_rn(make_float2(s0.x, s0.y), ntx);
                    dy = __fadd2_rn(make_float2(s0.z, s0.w), nty);
                } else {
                    s0 = __ldg(&slots[index]);
                    s1 = __ldg(&slots_b[index]);
                    const float2 sx = make_float2(shift_x[a], shift_x[a]);
                    const float2 sy = make_float2(shift_y, shift_y);
                    dx = __fadd2_rn(__fadd2_rn(make_float2(s0.x, s0.y), sx), ntx);
                    dy = __fadd2_rn(__fadd2_rn(make_float2(s0.z, s0.w), sy), nty);
                }
                pair_add2_gm(k, dx, dy, s1, ax2, ay2);
                continue;
            }
            const int count = __ldg(&cell_count[index]);
            if (count == 0) continue;
            if (!home && count > p.exact) {
                const float mass = (float)__ldg(&cell_mass[index]) * (1.0f / kCellMassUnits);
                const float dx = ((float)col[a] + 0.5f) * inv_w + shift_x[a] - t.x;
                float ax = ax2.x, ay = ay2.x;
                pair_add(k, dx, (cyr + shift_y) - t.y, mass, ax, ay);
                ax2.x = ax;
                ay2.x = ay;
            } else {
                // The list walk, two entries at a time.
                const int limit = home ? p.home_limit : p.exact;
                const int walk = count < limit ? count : limit;
                const int start = __ldg(&cell_start[index]);
                const float2 sx = make_float2(shift_x[a], shift_x[a]);
                const float2 sy = make_float2(shift_y, shift_y);
                for (int e = 0; e < walk; e += 2) {
                    const float4 o0 = __ldg(&entries[start + e]);
                    const bool has1 = e + 1 < walk;
                    const float4 o1 = has1 ? __ldg(&entries[start + e + 1]) : o0;
                    walk_step(k, o0, o1, has1, id, sx, sy, ntx, nty, ax2, ay2);
                }
            }
        }
    }
    acc_x = ax2;
    acc_y = ay2;
}

// Shared memory of the two-slot form (EXACT = 2): the staged slot-table box
// and the CTA's box reduction.
struct SlotStage {
    float4 a[kStageCells];
    float2 b[kStageCells];
    int red[4 * 32];
};

template <int RX, int RY, int EXACT>
__device__ __forceinline__ void short_range_body(
    SlotStage* sm, int block, const float4* __restrict__ bodies, const float4* __restrict__ entries,
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const uint32_t* __restrict__ cell_mass, const float4* __restrict__ slots,
    float2* __restrict__ a_short, const KickParams& p) {
    const int i = block * blockDim.x + threadIdx.x;
    const bool valid = i < p.n;
    if (EXACT != 2 && !valid) return;
    const float4 t = valid ? bodies[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const uint32_t id = (uint32_t)i;
    const PairConst k = pair_const(p);
    const float2* __restrict__ slots_b =
        reinterpret_cast<const float2*>(slots + (size_t)p.W * p.H);
    const int hx = guard_coord(float_to_int(floorf(t.x * (float)p.W)), p.W);
    const int hy = guard_coord(float_to_int(floorf(t.y * (float)p.H)), p.H);

    StageBox box{0, 0, 0, 0, false};
    HomeCell home{0, 0, make_float4(0.0f, 0.0f, 0.0f, 0.0f), make_float4(0.0f, 0.0f, 0.0f, 0.0f)};
    int sbase = 0;
    float4* st_a = nullptr;
    float2* st_b = nullptr;
    if (EXACT == 2) {
        st_a = sm->a;
        st_b = sm->b;
        // The home cell's count and start go out with the body; its first
        // two entries between the staging barriers. Their round trips then
        // overlap the staging instead of stalling the stencil.
        int count = 0;
        if (valid) {
            const int cell = hy * p.W + hx;
            count = __ldg(&cell_count[cell]);
            home.start = __ldg(&cell_start[cell]);
        }
        home.walk = count < p.home_limit ? count : p.home_limit;
        box = stage_box<RX, RY>(valid, hx, hy, sm->red);
        if (home.walk > 0) {
            home.e0 = __ldg(&entries[home.start]);
            home.e1 = home.walk > 1 ? __ldg(&entries[home.start + 1]) : home.e0;
        }
        stage_fill(box, slots, slots_b, p, sm->a, sm->b);
        if (!valid) return;
        if (box.staged) sbase = (hy - RY - box.y0) * box.w + (hx - RX - box.x0);
    }

    float2 acc_x, acc_y;
    if (EXACT == 2 && box.staged)
        stencil_sum<RX, RY, EXACT, true>(t, id, hx, hy, k, p, entries, cell_start, cell_count,
                                         cell_mass, slots, slots_b, st_a, st_b, sbase, box.w,
                                         home, acc_x, acc_y);
    else
        stencil_sum<RX, RY, EXACT, false>(t, id, hx, hy, k, p, entries, cell_start, cell_count,
                                          cell_mass, slots, slots_b, st_a, st_b, sbase, box.w,
                                          home, acc_x, acc_y);
    a_short[id] = make_float2(acc_x.x + acc_x.y, acc_y.x + acc_y.y);
}

template <int RX, int RY, int EXACT>
__global__ void __launch_bounds__(256, 4) short_range_kernel(
    const float4* __restrict__ bodies, const float4* __restrict__ entries,
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const uint32_t* __restrict__ cell_mass, const float4* __restrict__ slots,
    float2* __restrict__ a_short, KickParams p) {
    grid_dependency_wait();
    SlotStage* sm = nullptr;  // the two-slot form's stage; the list form has none
    if constexpr (EXACT == 2) {
        __shared__ SlotStage stage;
        sm = &stage;
    }
    short_range_body<RX, RY, EXACT>(sm, blockIdx.x, bodies, entries, cell_start, cell_count,
                                    cell_mass, slots, a_short, p);
}

template <int RX, int RY, int EXACT>
__global__ void __launch_bounds__(256, 4) short_range_batched_kernel(
    const ShortRangeArgs* __restrict__ args, const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const ShortRangeArgs a = args[sb.x];
    SlotStage* sm = nullptr;
    if constexpr (EXACT == 2) {
        __shared__ SlotStage stage;
        sm = &stage;
    }
    short_range_body<RX, RY, EXACT>(sm, sb.y, a.bodies, a.entries, a.cell_start, a.cell_count,
                                    a.cell_mass, a.slots, a.a_short, a.p);
}

}  // namespace sr

#ifndef P3M_COHERENT_BODIES
// Launches short_range_kernel<RX, p.ry, 2 or 0>; defined (explicitly
// instantiated) in p3m_short_range_rN.cu.
template <int RX>
cudaError_t launch_short_range_rx(const float4* bodies, const float4* entries,
                                  const int* cell_start, const int* cell_count,
                                  const uint32_t* cell_mass, const float4* slots, float2* a_short,
                                  const KickParams& p, cudaStream_t stream);
#define P3M_DECLARE_SHORT_RANGE_RX(RX_)                                                       \
    template <>                                                                                 \
    cudaError_t launch_short_range_rx<RX_>(const float4*, const float4*, const int*, const int*, \
                                           const uint32_t*, const float4*, float2*,             \
                                           const KickParams&, cudaStream_t);                    \
    template <>                                                                                 \
    cudaError_t batched_short_range_rx<RX_>(const ShortRangeArgs*, BatchGrid, int, int,          \
                                            cudaStream_t);
template <int RX>
cudaError_t batched_short_range_rx(const ShortRangeArgs* a, BatchGrid g, int ry, int exact2,
                                   cudaStream_t stream);
P3M_DECLARE_SHORT_RANGE_RX(1)
P3M_DECLARE_SHORT_RANGE_RX(2)
P3M_DECLARE_SHORT_RANGE_RX(3)
P3M_DECLARE_SHORT_RANGE_RX(4)
P3M_DECLARE_SHORT_RANGE_RX(5)
P3M_DECLARE_SHORT_RANGE_RX(6)
#undef P3M_DECLARE_SHORT_RANGE_RX

#define P3M_DEFINE_SHORT_RANGE_RX(RX_)                                                          \
    template <>                                                                                 \
    cudaError_t launch_short_range_rx<RX_>(const float4* bodies, const float4* entries,         \
                                           const int* cell_start, const int* cell_count,        \
                                           const uint32_t* cell_mass, const float4* slots,      \
                                           float2* a_short, const KickParams& p,                \
                                           cudaStream_t stream) {                               \
        const int threads_ = p.sr_threads > 0 ? p.sr_threads : 256;                               \
        const dim3 grid((p.n + threads_ - 1) / threads_), block(threads_);                      \
        switch (p.ry * 2 + (p.slot_form ? 1 : 0)) {                                             \
            case 3: launch_chained(sr::short_range_kernel<RX_, 1, 2>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 2: launch_chained(sr::short_range_kernel<RX_, 1, 0>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 5: launch_chained(sr::short_range_kernel<RX_, 2, 2>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 4: launch_chained(sr::short_range_kernel<RX_, 2, 0>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 7: launch_chained(sr::short_range_kernel<RX_, 3, 2>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 6: launch_chained(sr::short_range_kernel<RX_, 3, 0>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 9: launch_chained(sr::short_range_kernel<RX_, 4, 2>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 8: launch_chained(sr::short_range_kernel<RX_, 4, 0>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 11: launch_chained(sr::short_range_kernel<RX_, 5, 2>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 10: launch_chained(sr::short_range_kernel<RX_, 5, 0>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 13: launch_chained(sr::short_range_kernel<RX_, 6, 2>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            case 12: launch_chained(sr::short_range_kernel<RX_, 6, 0>, grid, block, 0, stream, bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p); break; \
            default: return cudaErrorInvalidValue;                                              \
        }                                                                                       \
        return cudaGetLastError();                                                              \
    }                                                                                           \
    template <>                                                                                 \
    cudaError_t batched_short_range_rx<RX_>(const ShortRangeArgs* a, BatchGrid g, int ry,       \
                                            int exact2, cudaStream_t stream) {                  \
        const dim3 grid(g.blocks), block(kBatchThreads);                                        \
        switch (ry * 2 + (exact2 ? 1 : 0)) {                                                    \
            case 3: sr::short_range_batched_kernel<RX_, 1, 2><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 2: sr::short_range_batched_kernel<RX_, 1, 0><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 5: sr::short_range_batched_kernel<RX_, 2, 2><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 4: sr::short_range_batched_kernel<RX_, 2, 0><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 7: sr::short_range_batched_kernel<RX_, 3, 2><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 6: sr::short_range_batched_kernel<RX_, 3, 0><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 9: sr::short_range_batched_kernel<RX_, 4, 2><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 8: sr::short_range_batched_kernel<RX_, 4, 0><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 11: sr::short_range_batched_kernel<RX_, 5, 2><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 10: sr::short_range_batched_kernel<RX_, 5, 0><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 13: sr::short_range_batched_kernel<RX_, 6, 2><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            case 12: sr::short_range_batched_kernel<RX_, 6, 0><<<grid, block, 0, stream>>>(a, g.first, g.sims); break; \
            default: return cudaErrorInvalidValue;                                              \
        }                                                                                       \
        return cudaGetLastError();                                                              \
    }

#endif  // !P3M_COHERENT_BODIES

}  // namespace p3m

#endif  // inclusion guard
