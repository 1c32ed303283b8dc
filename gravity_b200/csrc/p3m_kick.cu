// p3m_kick.cu — CIC force interpolation + short-range correction + half kick.
//
// Restates kick.comp:66-156: the mesh force is interpolated at the body with
// the CIC weights (kick.comp:82-103), the uniform field is added, and the
// short-range complement of the Gaussian split is summed over the
// (2Rx+1)x(2Ry+1) cell stencil around the home cell (kick.comp:122-151):
// cells holding more than `exact` bodies act as a monopole at the cell centre
// with the fixed-point cell mass; other cells, and the home cell up to
// `home_limit` list entries, are summed body by body in list order (the cell
// lists run in descending ID). Then v += a * dt/2 unless initial, and a is
// stored.
//
// The pair term G m exp(-r^2/2s^2) d / (M max(r^2, r_min^2)) is evaluated as
// (G/M) m exp2(-r^2 log2(e)/2s^2) * rcp(max(r^2, r_min^2)) * d: the same
// expression with fused multiply-adds, the hardware exp2 and a reciprocal
// instead of three IEEE divisions. Forces agree with the oracle's literal
// FP32 evaluation to ~1e-7 relative per term; the contract is 1e-5 relative
// RMS.
//
// One thread per body in ID order: after the Morton reorder, IDs follow
// screen tiles, so the stencils of a warp overlap and the cell tables and
// neighbour entries are served from L1/L2.

#include "p3m_internal.cuh"

namespace p3m {
namespace {

struct KickConst {
    float neg_log2e_over_2s2;  // -log2(e) / (2 sigma^2)
    float min_dist2;           // (min_frac * min(cell w, cell h))^2
    float g_over_m;            // G / M_tot
    float inv_w, inv_h;
};

__device__ __forceinline__ void pair_term(const KickParams& p, const KickConst& k, float sx,
                                          float sy, float tx, float ty, float m, float& ax,
                                          float& ay) {
    float dx = sx - tx, dy = sy - ty;
    if (p.bounded == 0) {
        dx -= floorf(dx + 0.5f);
        dy -= floorf(dy + 0.5f);
    }
    const float px = dx * p.aspect;
    const float r2 = fmaf(px, px, dy * dy);
    const float w = exp2f(r2 * k.neg_log2e_over_2s2);
    const float phys = __fdividef(k.g_over_m * m * w, fmaxf(r2, k.min_dist2));
    // (phys * px) / aspect == phys * dx
    ax = fmaf(phys, dx, ax);
    ay = fmaf(phys, dy, ay);
}

__global__ void __launch_bounds__(256) kick_kernel(
    float4* __restrict__ bodies, float2* __restrict__ accel, const float2* __restrict__ force,
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const uint32_t* __restrict__ cell_mass, const float4* __restrict__ entries, KickParams p) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= p.n) return;
    float4 b = bodies[id];
    if (p.mutual == 0) {
        // Field only: the same separately rounded multiply and add as the
        // oracle (this file otherwise allows contraction).
        if (p.initial == 0) {
            b.z = __fadd_rn(b.z, __fmul_rn(p.field_x, 0.5f * p.dt));
            b.w = __fadd_rn(b.w, __fmul_rn(p.field_y, 0.5f * p.dt));
        }
        accel[id] = make_float2(p.field_x, p.field_y);
        bodies[id] = b;
        return;
    }
    KickConst k;
    {
        const float sigma = p.sigma_cells / (float)p.H;
        k.neg_log2e_over_2s2 = -1.4426950408889634f / (2.0f * sigma * sigma);
        const float cw = p.aspect / (float)p.W, ch = 1.0f / (float)p.H;
        const float md = p.min_frac * fminf(cw, ch);
        k.min_dist2 = md * md;
        k.g_over_m = p.gravity / p.total_mass;
        k.inv_w = 1.0f / (float)p.W;
        k.inv_h = 1.0f / (float)p.H;
    }
    // kick.comp:82-103 interpolateForce.
    float rx, ry;
    {
        const float gx = b.x * (float)p.W - 0.5f, gy = b.y * (float)p.H - 0.5f;
        const float flx = floorf(gx), fly = floorf(gy);
        const int bx = guard_coord(float_to_int(flx), p.MW), by = guard_coord(float_to_int(fly), p.MH);
        const float tx = gx - flx, ty = gy - fly;
        const int x0 = wrap_index(bx, p.MW), x1 = wrap_index(bx + 1, p.MW);
        const int y0 = wrap_index(by, p.MH), y1 = wrap_index(by + 1, p.MH);
        const float2 v00 = __ldg(&force[(size_t)y0 * p.MW + x0]);
        const float2 v10 = __ldg(&force[(size_t)y0 * p.MW + x1]);
        const float2 v01 = __ldg(&force[(size_t)y1 * p.MW + x0]);
        const float2 v11 = __ldg(&force[(size_t)y1 * p.MW + x1]);
        const float ax = v00.x * (1.0f - tx) + v10.x * tx;
        const float ay = v00.y * (1.0f - tx) + v10.y * tx;
        const float bx2 = v01.x * (1.0f - tx) + v11.x * tx;
        const float by2 = v01.y * (1.0f - tx) + v11.y * tx;
        rx = ax * (1.0f - ty) + bx2 * ty + p.field_x;
        ry = ay * (1.0f - ty) + by2 * ty + p.field_y;
    }

    const int hx = guard_coord(float_to_int(floorf(b.x * (float)p.W)), p.W);
    const int hy = guard_coord(float_to_int(floorf(b.y * (float)p.H)), p.H);
    for (int dy = -p.ry; dy <= p.ry; ++dy) {
        const int cy = hy + dy;
        if (p.bounded && (cy < 0 || cy >= p.H)) continue;
        const int wy = wrap_index(cy, p.H);
        const int row = wy * p.W;
        const float cyf = ((float)wy + 0.5f) * k.inv_h;
        for (int dx = -p.rx; dx <= p.rx; ++dx) {
            const int cx = hx + dx;
            if (p.bounded && (cx < 0 || cx >= p.W)) continue;
            const int wx = wrap_index(cx, p.W);
            const int index = wx + row;
            const int count = __ldg(&cell_count[index]);
            if (count == 0) continue;
            const bool home = dx == 0 && dy == 0;
            if (!home && count > p.exact) {
                const float cxf = ((float)wx + 0.5f) * k.inv_w;
                const float agg = (float)__ldg(&cell_mass[index]) * (1.0f / kCellMassUnits);
                pair_term(p, k, cxf, cyf, b.x, b.y, agg, rx, ry);
            } else {
                const int limit = home ? p.home_limit : p.exact;
                const int walk = count < limit ? count : limit;
                const int start = __ldg(&cell_start[index]);
                for (int e = 0; e < walk; ++e) {
                    const float4 o = __ldg(&entries[start + e]);
                    if (__float_as_uint(o.w) != (uint32_t)id)
                        pair_term(p, k, o.x, o.y, b.x, b.y, o.z, rx, ry);
                }
            }
        }
    }
    if (p.initial == 0) {
        b.z = __fadd_rn(b.z, __fmul_rn(rx, 0.5f * p.dt));
        b.w = __fadd_rn(b.w, __fmul_rn(ry, 0.5f * p.dt));
    }
    accel[id] = make_float2(rx, ry);
    bodies[id] = b;
}

}  // namespace

cudaError_t launch_kick(float4* bodies, float2* accel, const float2* force, const int* cell_start,
                        const int* cell_count, const uint32_t* cell_mass, const float4* entries,
                        KickParams p, cudaStream_t stream) {
    if (p.n <= 0) return cudaSuccess;
    kick_kernel<<<(p.n + 255) / 256, 256, 0, stream>>>(bodies, accel, force, cell_start,
                                                       cell_count, cell_mass, entries, p);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace p3m
