// p3m_trajectory.cu — aim previews on the P3M field (trajectory.comp).
//
// The reference integrates one test particle per call in a one-thread
// dispatch (trajectory.comp:262-329, GravityPipeline.kt:514-600): adaptive
// kick-drift-kick steps through the frozen field of the last force build
// (mesh force + the short-range stencil over the cell lists), emitting six
// line vertices per step, split where the path wraps (emitPeriodicStep,
// :178-260).
//
// Here one warp integrates one preview and many previews run in one launch
// (a fan of launch velocities, or previews for several origins). The step
// itself is sequential; the 49 stencil cells of accelerationAt (:120-163)
// are split over the lanes and their sums reduced across the warp, lane 0
// emitting the vertices. The arithmetic is the shader's (expf, IEEE
// division, the minimum image by rounding, lists in their walk order), built
// without contracted multiply-adds: the adaptive step length
// (sqrt(s^2 + 2 a L) - s) / a cancels, and a fused rounding there moves the
// whole path by ~1e-4. Only the order in which the stencil cells' terms are
// added differs from the shader.

#include "p3m_internal.cuh"

namespace p3m {
namespace {

// One preview (one warp) per CTA: a fan of a few hundred previews then
// spreads over every SM instead of sharing a quarter of them.
constexpr int kWarpsPerBlock = 1;
constexpr int kVerticesPerStep = 6;  // GravityPipeline.kt:1623

struct TrajParams {
    KickParams k;        // grid, radii, limits, gravity, field (unit/s^2), mutual, bounded
    float2 viewport;     // px
    float min_dt, max_dt, target_segment_px, max_path_px, min_dash_px, restitution;
    int steps;
};

// localAcceleration (trajectory.comp:78-95).
__device__ __forceinline__ float2 local_acceleration(const TrajParams& P, float2 src, float2 tgt,
                                                      float m) {
    float dx = src.x - tgt.x, dy = src.y - tgt.y;
    if (P.k.bounded == 0) {
        dx -= floorf(dx + 0.5f);
        dy -= floorf(dy + 0.5f);
    }
    const float px = dx * P.k.aspect, py = dy;
    const float r2 = px * px + py * py;
    const float sigma = P.k.sigma_cells / (float)P.k.H;
    const float w = expf(-r2 / (2.0f * sigma * sigma));
    const float cw = P.k.aspect / (float)P.k.W, ch = 1.0f / (float)P.k.H;
    const float md = P.k.min_frac * fminf(cw, ch);
    const float phys = P.k.gravity * m * w / (P.k.total_mass * fmaxf(r2, md * md));
    return make_float2(phys * px / P.k.aspect, phys * py);
}

// accelerationAt (trajectory.comp:120-163): every lane returns the total.
// A preview is one chain of dependent steps, so this is latency: the mesh
// force's four taps are loaded first, and each lane's cells (c, c + 32, ...)
// are taken two at a time with their count, start and mass loaded together,
// so the stencil waits on fewer round trips. The arithmetic and its order
// are those of one cell after the other.
__device__ float2 acceleration_at(const TrajParams& P, float2 pos, const float2* __restrict__ force,
                                  const float4* __restrict__ entries,
                                  const int* __restrict__ cell_start,
                                  const int* __restrict__ cell_count,
                                  const uint32_t* __restrict__ cell_mass) {
    const KickParams& k = P.k;
    if (k.mutual == 0) return make_float2(k.field_x, k.field_y);
    const int lane = threadIdx.x & 31;
    // interpolateForce's taps (:97-118).
    const float gx = pos.x * (float)k.W - 0.5f, gy = pos.y * (float)k.H - 0.5f;
    const float flx = floorf(gx), fly = floorf(gy);
    const int bx = guard_coord(float_to_int(flx), k.MW), by = guard_coord(float_to_int(fly), k.MH);
    const float tx = gx - flx, ty = gy - fly;
    const int x0 = wrap_index(bx, k.MW), x1 = wrap_index(bx + 1, k.MW);
    const int y0 = wrap_index(by, k.MH), y1 = wrap_index(by + 1, k.MH);
    const float2 v00 = __ldg(&force[(size_t)y0 * k.MW + x0]);
    const float2 v10 = __ldg(&force[(size_t)y0 * k.MW + x1]);
    const float2 v01 = __ldg(&force[(size_t)y1 * k.MW + x0]);
    const float2 v11 = __ldg(&force[(size_t)y1 * k.MW + x1]);

    float ax = 0.0f, ay = 0.0f;
    const int sx = 2 * k.rx + 1, cells = sx * (2 * k.ry + 1);
    const int hx = guard_coord(float_to_int(floorf(pos.x * (float)k.W)), k.W);
    const int hy = guard_coord(float_to_int(floorf(pos.y * (float)k.H)), k.H);
    for (int base = lane; base < cells; base += 64) {
        int index[2], wxs[2], wys[2], count[2], start[2];
        uint32_t mass[2];
        bool ok[2], home[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int c = base + 32 * j;
            const int dy = c / sx - k.ry, dx = c % sx - k.rx;
            const int cx = hx + dx, cy = hy + dy;
            ok[j] = c < cells && !(k.bounded != 0 && (cx < 0 || cy < 0 || cx >= k.W || cy >= k.H));
            home[j] = dx == 0 && dy == 0;
            wxs[j] = wrap_index(cx, k.W);
            wys[j] = wrap_index(cy, k.H);
            index[j] = wxs[j] + wys[j] * k.W;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            count[j] = ok[j] ? __ldg(&cell_count[index[j]]) : 0;
            start[j] = ok[j] ? __ldg(&cell_start[index[j]]) : 0;
            mass[j] = ok[j] ? __ldg(&cell_mass[index[j]]) : 0u;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (!ok[j]) continue;
            if (!home[j] && count[j] > k.exact) {
                const float2 center = make_float2(((float)wxs[j] + 0.5f) / (float)k.W,
                                                  ((float)wys[j] + 0.5f) / (float)k.H);
                const float2 a = local_acceleration(P, center, pos, (float)mass[j] / kCellMassUnits);
                ax += a.x;
                ay += a.y;
            } else if (count[j] > 0) {
                const int limit = home[j] ? k.home_limit : k.exact;
                const int walk = count[j] < limit ? count[j] : limit;
                const float4 o0 = __ldg(&entries[start[j]]);
                const float4 o1 = walk > 1 ? __ldg(&entries[start[j] + 1]) : o0;
                for (int e = 0; e < walk; ++e) {
                    const float4 o = e == 0 ? o0 : (e == 1 ? o1 : __ldg(&entries[start[j] + e]));
                    const float2 a = local_acceleration(P, make_float2(o.x, o.y), pos, o.z);
                    ax += a.x;
                    ay += a.y;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    // Every lane holds the same sum (IEEE addition commutes); lane 0's is
    // taken anyway so that the lanes' step decisions cannot part.
    ax = __shfl_sync(0xffffffffu, ax, 0);
    ay = __shfl_sync(0xffffffffu, ay, 0);
    // The interpolated force + the field, then the stencil sum.
    const float lx = v00.x * (1.0f - tx) + v10.x * tx, ly = v00.y * (1.0f - tx) + v10.y * tx;
    const float ux = v01.x * (1.0f - tx) + v11.x * tx, uy = v01.y * (1.0f - tx) + v11.y * tx;
    float2 r;
    r.x = (lx * (1.0f - ty) + ux * ty + k.field_x) + ax;
    r.y = (ly * (1.0f - ty) + uy * ty + k.field_y) + ay;
    return r;
}

__device__ __forceinline__ float integration_dt(const TrajParams& P, float2 v, float2 a) {
    const float speed = sqrtf((v.x * P.viewport.x) * (v.x * P.viewport.x) +
                              (v.y * P.viewport.y) * (v.y * P.viewport.y));
    const float accel = sqrtf((a.x * P.viewport.x) * (a.x * P.viewport.x) +
                              (a.y * P.viewport.y) * (a.y * P.viewport.y));
    float r;
    if (accel > 1e-5f) r = (sqrtf(speed * speed + 2.0f * accel * P.target_segment_px) - speed) / accel;
    else r = P.target_segment_px / fmaxf(speed, 1e-5f);
    return fminf(fmaxf(r, P.min_dt), P.max_dt);
}

// emitPeriodicStep (:178-260), by one lane.
__device__ void emit_step(float4* __restrict__ out, int step, float2 start, float2 delta,
                          float start_distance, float step_distance, float start_dash,
                          float step_dash) {
    float4* v = out + (size_t)step * kVerticesPerStep;
    for (int i = 0; i < kVerticesPerStep; ++i) v[i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    const float2 end = make_float2(start.x + delta.x, start.y + delta.y);
    float cuts[4];
    int cut_count = 2;
    cuts[0] = 0.0f;
    cuts[1] = 1.0f;
    if (end.x < 0.0f) cuts[cut_count++] = -start.x / delta.x;
    else if (end.x >= 1.0f) cuts[cut_count++] = (1.0f - start.x) / delta.x;
    if (end.y < 0.0f) cuts[cut_count++] = -start.y / delta.y;
    else if (end.y >= 1.0f) cuts[cut_count++] = (1.0f - start.y) / delta.y;
    for (int index = 1; index < cut_count; ++index) {
        const float value = fminf(fmaxf(cuts[index], 0.0f), 1.0f);
        int insertion = index;
        while (insertion > 0 && cuts[insertion - 1] > value) {
            cuts[insertion] = cuts[insertion - 1];
            insertion--;
        }
        cuts[insertion] = value;
    }
    float unique[4];
    int unique_count = 0;
    for (int index = 0; index < cut_count; ++index)
        if (unique_count == 0 || fabsf(cuts[index] - unique[unique_count - 1]) > 1e-6f)
            unique[unique_count++] = cuts[index];
    for (int piece = 0; piece < unique_count - 1; ++piece) {
        const float f0 = unique[piece], f1 = unique[piece + 1];
        const float mid = 0.5f * (f0 + f1);
        const float tile_x = floorf(start.x + delta.x * mid), tile_y = floorf(start.y + delta.y * mid);
        const float ax_ = start.x + delta.x * f0 - tile_x, ay_ = start.y + delta.y * f0 - tile_y;
        const float bx_ = start.x + delta.x * f1 - tile_x, by_ = start.y + delta.y * f1 - tile_y;
        v[piece * 2] = make_float4(fminf(fmaxf(ax_, 0.0f), 1.0f), fminf(fmaxf(ay_, 0.0f), 1.0f),
                                   start_dash + step_dash * f0, start_distance + step_distance * f0);
        v[piece * 2 + 1] = make_float4(fminf(fmaxf(bx_, 0.0f), 1.0f), fminf(fmaxf(by_, 0.0f), 1.0f),
                                       start_dash + step_dash * f1,
                                       start_distance + step_distance * f1);
    }
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock) trajectory_kernel(
    TrajParams P, int count, const float2* __restrict__ origins_px,
    const float2* __restrict__ velocities_px, const float2* __restrict__ force,
    const float4* __restrict__ entries, const int* __restrict__ cell_start,
    const int* __restrict__ cell_count, const uint32_t* __restrict__ cell_mass,
    float4* __restrict__ vertices) {
    const int preview = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    if (preview >= count) return;  // whole warps leave together
    const int lane = threadIdx.x & 31;
    float4* out = vertices + (size_t)preview * P.steps * kVerticesPerStep;
    float2 o = origins_px[preview];
    const float2 vp = velocities_px[preview];
    // placeX / placeY (GravityPipeline.kt:773-779, ToroidalSpace.kt:11-14).
    if (P.k.bounded != 0) {
        o.x = fminf(fmaxf(o.x, 0.0f), P.viewport.x * kMaximumUnit);
        o.y = fminf(fmaxf(o.y, 0.0f), P.viewport.y * kMaximumUnit);
    } else {
        o.x = o.x - floorf(o.x / P.viewport.x) * P.viewport.x;
        o.y = o.y - floorf(o.y / P.viewport.y) * P.viewport.y;
    }
    float2 pos = make_float2(o.x / P.viewport.x, o.y / P.viewport.y);
    float2 vel = make_float2(vp.x / P.viewport.x, vp.y / P.viewport.y);
    float2 acc = acceleration_at(P, pos, force, entries, cell_start, cell_count, cell_mass);
    float path = 0.0f, dash = 0.0f;
    bool finished = false;
    for (int step = 0; step < P.steps; ++step) {
        if (finished) {
            if (lane == 0)
                for (int i = 0; i < kVerticesPerStep; ++i)
                    out[(size_t)step * kVerticesPerStep + i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
            continue;
        }
        const float dt = integration_dt(P, vel, acc);
        float2 half = make_float2(vel.x + acc.x * (0.5f * dt), vel.y + acc.y * (0.5f * dt));
        float2 delta = make_float2(half.x * dt, half.y * dt);
        if (P.k.bounded != 0) {
            // A wall is treated as a contact: the velocity component into
            // the wall is reflected and scaled by the restitution
            // coefficient (0 stops it).
            const float nx = pos.x + delta.x, ny = pos.y + delta.y;
            const float cx = fminf(fmaxf(nx, 0.0f), kMaximumUnit);
            const float cy = fminf(fmaxf(ny, 0.0f), kMaximumUnit);
            if (nx != cx) half.x = -P.restitution * half.x;
            if (ny != cy) half.y = -P.restitution * half.y;
            delta = make_float2(cx - pos.x, cy - pos.y);
        }
        float step_px = sqrtf((delta.x * P.viewport.x) * (delta.x * P.viewport.x) +
                              (delta.y * P.viewport.y) * (delta.y * P.viewport.y));
        const float remaining = P.max_path_px - path;
        if (step_px > remaining) {
            delta.x *= remaining / step_px;
            delta.y *= remaining / step_px;
            step_px = remaining;
            finished = true;
        }
        const float speed_multiplier = 1.0f + sqrtf(half.x * half.x + half.y * half.y);
        const float dash_len = P.min_dash_px * speed_multiplier;
        const float step_dash = step_px * P.min_dash_px / dash_len;
        if (lane == 0) emit_step(out, step, pos, delta, path, step_px, dash, step_dash);
        path += step_px;
        dash += step_dash;
        if (P.k.bounded != 0) pos = make_float2(pos.x + delta.x, pos.y + delta.y);
        else {
            const float px = pos.x + delta.x, py = pos.y + delta.y;
            pos = make_float2(px - floorf(px), py - floorf(py));
        }
        if (path >= P.max_path_px - 1e-4f) {
            finished = true;
            continue;
        }
        acc = acceleration_at(P, pos, force, entries, cell_start, cell_count, cell_mass);
        vel = make_float2(half.x + acc.x * (0.5f * dt), half.y + acc.y * (0.5f * dt));
    }
    __syncwarp();
    // Distances along the path, normalised (:321-328).
    const float inverse = 1.0f / fmaxf(path, 1e-6f);
    for (int v = lane; v < P.steps * kVerticesPerStep; v += 32) {
        float4 q = out[v];
        if (q.w >= 0.0f) {
            q.w = fminf(fmaxf(q.w * inverse, 0.0f), 1.0f);
            out[v] = q;
        }
    }
}

}  // namespace

cudaError_t launch_trajectories(const KickParams& k, float2 viewport, float min_dt, float max_dt,
                                float target_segment_px, float max_path_px, float min_dash_px,
                                float restitution, int steps, int count, const float2* origins_px,
                                const float2* velocities_px, const float2* force,
                                const float4* entries, const int* cell_start,
                                const int* cell_count, const uint32_t* cell_mass,
                                float4* vertices, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    TrajParams P;
    P.k = k;
    P.viewport = viewport;
    P.min_dt = min_dt;
    P.max_dt = max_dt;
    P.target_segment_px = target_segment_px;
    P.max_path_px = max_path_px;
    P.min_dash_px = min_dash_px;
    P.restitution = restitution;
    P.steps = steps;
    const int blocks = (count + kWarpsPerBlock - 1) / kWarpsPerBlock;
    trajectory_kernel<<<blocks, 32 * kWarpsPerBlock, 0, stream>>>(
        P, count, origins_px, velocities_px, force, entries, cell_start, cell_count, cell_mass,
        vertices);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace p3m
