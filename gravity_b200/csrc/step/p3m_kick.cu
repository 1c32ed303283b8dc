// p3m_kick.cu — CIC force interpolation + half kick, and the short-range
// dispatch.
//
// kick.comp:66-156 runs here as two kernels: the short-range correction
// (p3m_short_range.cuh, one instantiation per stencil size) writes a_short[id];
// then interp_kick, one thread per body in ID order (coalesced state), adds
// the CIC interpolation of the mesh force (kick.comp:82-103), the uniform
// field and a_short, and applies v += a * dt/2 unless initial, storing a
// (kick.comp:153-154). interp_kick streams bodies and the force mesh once, so
// it runs near the HBM roofline on its own.

#include "p3m_short_range.cuh"

namespace p3m {
namespace {

__device__ __forceinline__ void interp_kick_body(
    int block, float4* __restrict__ bodies, float2* __restrict__ accel,
    const float2* __restrict__ force, const float2* __restrict__ a_short, const KickParams& p) {
    const int id = block * blockDim.x + threadIdx.x;
    if (id >= p.n) return;
    float4 b = bodies[id];
    float rx, ry;
    if (p.mutual == 0) {
        rx = p.field_x;
        ry = p.field_y;
    } else {
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
        const float lx = v00.x * (1.0f - tx) + v10.x * tx;
        const float ly = v00.y * (1.0f - tx) + v10.y * tx;
        const float ux = v01.x * (1.0f - tx) + v11.x * tx;
        const float uy = v01.y * (1.0f - tx) + v11.y * tx;
        const float2 s = __ldg(&a_short[id]);
        rx = (lx * (1.0f - ty) + ux * ty + p.field_x) + s.x;
        ry = (ly * (1.0f - ty) + uy * ty + p.field_y) + s.y;
    }
    // The velocity update rounds like the oracle's separate multiply and add
    // (this file otherwise allows contraction).
    if (p.initial == 0) {
        b.z = __fadd_rn(b.z, __fmul_rn(rx, 0.5f * p.dt));
        b.w = __fadd_rn(b.w, __fmul_rn(ry, 0.5f * p.dt));
    }
    accel[id] = make_float2(rx, ry);
    bodies[id] = b;
}

__global__ void __launch_bounds__(256) interp_kick_kernel(
    float4* __restrict__ bodies, float2* __restrict__ accel, const float2* __restrict__ force,
    const float2* __restrict__ a_short, KickParams p) {
    grid_dependency_wait();
    interp_kick_body(blockIdx.x, bodies, accel, force, a_short, p);
}

// One thread per cell: the two source slots the two-slot short range reads
// for a non-home cell (kick.comp:128-146 with exact limit 2). A cell of more
// than two bodies is its monopole at the cell centre; one of up to two bodies
// gives its entries; missing slots are massless at the centre, so they add
// nothing. The short range then reads 24 bytes per cell instead of the
// count -> start -> entries chain. A slot holds x, y and G m / M_tot, the
// product the pair term forms first; the two slots of a cell are stored
// interleaved, (x0, x1, y0, y1) and (G m0 / M, G m1 / M).
__device__ __forceinline__ void cell_slots_body(
    int block, const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const uint32_t* __restrict__ cell_mass, const float4* __restrict__ entries, int W, int H,
    float gravity, float total_mass, float4* __restrict__ slots) {
    const int index = block * blockDim.x + threadIdx.x;
    if (index >= W * H) return;
    const int row = index / W, col = index - row * W;
    const float inv_w = 1.0f / (float)W, inv_h = 1.0f / (float)H;
    float4 s0 = make_float4(((float)col + 0.5f) * inv_w, ((float)row + 0.5f) * inv_h, 0.0f, 0.0f);
    float4 s1 = s0;
    // The count, start and mass loads are independent: issued together, the
    // entries wait on one round trip instead of two.
    const int count = cell_count[index];
    const int start = cell_start[index];
    const uint32_t mass = cell_mass[index];
    if (count > 2) {
        s0.z = (float)mass * (1.0f / kCellMassUnits);
    } else if (count > 0) {
        s0 = entries[start];
        if (count == 2) s1 = entries[start + 1];
    }
    const float g_over_m = gravity / total_mass;
    // Two planes: (x0, x1, y0, y1) for every cell, then (gm0, gm1), so that
    // each pair the packed FP32x2 pair term takes is loaded as one pair.
    slots[index] = make_float4(s0.x, s1.x, s0.y, s1.y);
    reinterpret_cast<float2*>(slots + (size_t)W * H)[index] =
        make_float2(g_over_m * s0.z, g_over_m * s1.z);
}

__global__ void __launch_bounds__(256) cell_slots_kernel(
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const uint32_t* __restrict__ cell_mass, const float4* __restrict__ entries, int W, int H,
    float gravity, float total_mass, float4* __restrict__ slots) {
    grid_dependency_wait();
    cell_slots_body(blockIdx.x, cell_start, cell_count, cell_mass, entries, W, H, gravity,
                    total_mass, slots);
}

__global__ void __launch_bounds__(256) cell_slots_batched_kernel(
    const SlotsArgs* __restrict__ args, const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const SlotsArgs a = args[sb.x];
    cell_slots_body(sb.y, a.cell_start, a.cell_count, a.cell_mass, a.entries, a.W, a.H,
                    a.gravity, a.total_mass, a.slots);
}

__global__ void __launch_bounds__(256) interp_kick_batched_kernel(
    const KickArgs* __restrict__ args, const int* __restrict__ first, int sims) {
    const int2 sb = batch_block(first, sims);
    const KickArgs a = args[sb.x];
    interp_kick_body(sb.y, a.bodies, a.accel, a.force, a.a_short, a.p);
}

}  // namespace

// Host-side launchers: not part of the coherent copy of the bodies that the
// batched form's persistent kernel uses (p3m_step.cu).
#ifndef P3M_COHERENT_BODIES

cudaError_t batched_interp_kick(const KickArgs* a, BatchGrid g, cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    interp_kick_batched_kernel<<<g.blocks, kBatchThreads, 0, s>>>(a, g.first, g.sims);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_cell_slots(const int* cell_start, const int* cell_count,
                              const uint32_t* cell_mass, const float4* entries, int W, int H,
                              float gravity, float total_mass, float4* slots,
                              cudaStream_t stream) {
    const int cells = W * H;
    if (cells <= 0) return cudaSuccess;
    launch_chained(cell_slots_kernel, (cells + 255) / 256, 256, 0, stream,
        cell_start, cell_count, cell_mass, entries, W, H, gravity, total_mass, slots);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t batched_cell_slots(const SlotsArgs* a, BatchGrid g, cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    cell_slots_batched_kernel<<<g.blocks, kBatchThreads, 0, s>>>(a, g.first, g.sims);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t batched_short_range(const ShortRangeArgs* a, BatchGrid g, int rx, int ry, int exact2,
                                cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    cudaError_t e;
    switch (rx) {
        case 1: e = batched_short_range_rx<1>(a, g, ry, exact2, s); break;
        case 2: e = batched_short_range_rx<2>(a, g, ry, exact2, s); break;
        case 3: e = batched_short_range_rx<3>(a, g, ry, exact2, s); break;
        case 4: e = batched_short_range_rx<4>(a, g, ry, exact2, s); break;
        case 5: e = batched_short_range_rx<5>(a, g, ry, exact2, s); break;
        case 6: e = batched_short_range_rx<6>(a, g, ry, exact2, s); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return e;
}

cudaError_t launch_short_range(const float4* bodies, const float4* entries, const int* cell_start,
                               const int* cell_count, const uint32_t* cell_mass,
                               const float4* slots, float2* a_short, KickParams p,
                               cudaStream_t stream) {
    if (p.n <= 0 || p.mutual == 0) return cudaSuccess;
    cudaError_t e;
    switch (p.rx) {
        case 1: e = launch_short_range_rx<1>(bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p, stream); break;
        case 2: e = launch_short_range_rx<2>(bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p, stream); break;
        case 3: e = launch_short_range_rx<3>(bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p, stream); break;
        case 4: e = launch_short_range_rx<4>(bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p, stream); break;
        case 5: e = launch_short_range_rx<5>(bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p, stream); break;
        case 6: e = launch_short_range_rx<6>(bodies, entries, cell_start, cell_count, cell_mass, slots, a_short, p, stream); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return e;
}

cudaError_t launch_interp_kick(float4* bodies, float2* accel, const float2* force,
                               const float2* a_short, KickParams p, cudaStream_t stream) {
    if (p.n <= 0) return cudaSuccess;
    launch_chained(interp_kick_kernel, (p.n + 255) / 256, 256, 0, stream, bodies, accel, force, a_short, p);
    count_launches(1);
    return cudaGetLastError();
}

#endif  // !P3M_COHERENT_BODIES
}  // namespace p3m
