// p3m_kick.cu — leapfrog drift and the interpolation + short-range + kick.
//
// Built with --fmad=false: every multiply and add rounds on its own, as in
// the oracle, so positions, keys and deposit weights derived from them are
// bit-identical to it.
//
// drift: collision_build.comp:40-51 (gravity-only, so only the half kick,
//   drift and wall clamp / torus wrap of each collision substep), all S
//   substeps in registers, then the home-cell key of the cell sort.
// kick:  kick.comp:66-156 — CIC interpolation of the mesh force, uniform
//   field, and the short-range correction over the (2Rx+1)x(2Ry+1) cell
//   stencil: exact pairs for cells with at most `exact` bodies (the home cell
//   walks at most `home_limit` list entries), a cell monopole otherwise; then
//   v += a * dt/2 unless initial, and a is stored.

#include "p3m_internal.cuh"

namespace p3m {
namespace {

__device__ __forceinline__ float fractf(float v) { return v - floorf(v); }

__global__ void drift_kernel(float4* __restrict__ bodies, const float2* __restrict__ accel, int n,
                             float half_kick, float drift_dt, int substeps, int bounded, int W,
                             int H, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                             unsigned int* __restrict__ nonfinite) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    float4 b = bodies[id];
    const float2 a = accel[id];
    for (int s = 0; s < substeps; ++s) {
        // Substeps after the first carry kickDt = 0 (GravityPipeline.kt:465-473),
        // whose kick adds a * 0.
        const float hk = s == 0 ? half_kick : 0.0f;
        b.z = b.z + a.x * hk;
        b.w = b.w + a.y * hk;
        b.x = b.x + b.z * drift_dt;
        b.y = b.y + b.w * drift_dt;
        if (bounded) {
            b.x = fminf(fmaxf(b.x, 0.0f), kMaximumUnit);
            b.y = fminf(fmaxf(b.y, 0.0f), kMaximumUnit);
        } else {
            b.x = fractf(b.x);
            b.y = fractf(b.y);
        }
    }
    bodies[id] = b;
    if (nonfinite && !(isfinite(b.x) && isfinite(b.y) && isfinite(b.z) && isfinite(b.w)))
        atomicAdd(nonfinite, 1u);
    if (keys) {
        const int hx = wrap_index(float_to_int(floorf(b.x * (float)W)), W);
        const int hy = wrap_index(float_to_int(floorf(b.y * (float)H)), H);
        const int slot = n - 1 - id;  // descending ID order for the cell sort
        keys[slot] = (uint32_t)hx + (uint32_t)hy * (uint32_t)W;
        vals[slot] = (uint32_t)id;
    }
}

struct KickConst {
    float sigma2x2;     // 2 sigma^2
    float min_dist2;    // (min_frac * min(cell w, cell h))^2
};

// kick.comp:66-80 localAcceleration.
__device__ __forceinline__ float2 local_acceleration(const KickParams& p, const KickConst& k,
                                                     float sx, float sy, float tx, float ty,
                                                     float m) {
    float dx = sx - tx, dy = sy - ty;
    if (p.bounded == 0) {
        dx -= floorf(dx + 0.5f);
        dy -= floorf(dy + 0.5f);
    }
    const float px = dx * p.aspect, py = dy;
    const float r2 = px * px + py * py;
    const float w = expf(-r2 / k.sigma2x2);
    const float phys = p.gravity * m * w / (p.total_mass * fmaxf(r2, k.min_dist2));
    return make_float2(phys * px / p.aspect, phys * py);
}

__global__ void __launch_bounds__(256) kick_kernel(
    float4* __restrict__ bodies, float2* __restrict__ accel, const float2* __restrict__ force,
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const uint32_t* __restrict__ cell_mass, const float4* __restrict__ entries, KickParams p) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= p.n) return;
    float4 b = bodies[id];
    if (p.mutual == 0) {
        if (p.initial == 0) {
            b.z = b.z + p.field_x * (0.5f * p.dt);
            b.w = b.w + p.field_y * (0.5f * p.dt);
        }
        accel[id] = make_float2(p.field_x, p.field_y);
        bodies[id] = b;
        return;
    }
    KickConst k;
    {
        const float sigma = p.sigma_cells / (float)p.H;
        k.sigma2x2 = 2.0f * sigma * sigma;
        const float cw = p.aspect / (float)p.W, ch = 1.0f / (float)p.H;
        const float md = p.min_frac * fminf(cw, ch);
        k.min_dist2 = md * md;
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
        rx = ax * (1.0f - ty) + bx2 * ty;
        ry = ay * (1.0f - ty) + by2 * ty;
    }
    rx = rx + p.field_x;
    ry = ry + p.field_y;

    const int hx = guard_coord(float_to_int(floorf(b.x * (float)p.W)), p.W);
    const int hy = guard_coord(float_to_int(floorf(b.y * (float)p.H)), p.H);
    for (int dy = -p.ry; dy <= p.ry; ++dy) {
        const int cy = hy + dy;
        if (p.bounded && (cy < 0 || cy >= p.H)) continue;
        const int wy = wrap_index(cy, p.H);
        for (int dx = -p.rx; dx <= p.rx; ++dx) {
            const int cx = hx + dx;
            if (p.bounded && (cx < 0 || cx >= p.W)) continue;
            const int wx = wrap_index(cx, p.W);
            const int index = wx + wy * p.W;
            const int count = __ldg(&cell_count[index]);
            if (count == 0) continue;
            const bool home = dx == 0 && dy == 0;
            if (!home && count > p.exact) {
                const float cxf = ((float)wx + 0.5f) / (float)p.W;
                const float cyf = ((float)wy + 0.5f) / (float)p.H;
                const float agg = (float)__ldg(&cell_mass[index]) / kCellMassUnits;
                const float2 a = local_acceleration(p, k, cxf, cyf, b.x, b.y, agg);
                rx = rx + a.x;
                ry = ry + a.y;
            } else {
                const int limit = home ? p.home_limit : p.exact;
                const int walk = count < limit ? count : limit;
                const int start = __ldg(&cell_start[index]);
                for (int e = 0; e < walk; ++e) {
                    const float4 o = __ldg(&entries[start + e]);
                    if (__float_as_uint(o.w) != (uint32_t)id) {
                        const float2 a = local_acceleration(p, k, o.x, o.y, b.x, b.y, o.z);
                        rx = rx + a.x;
                        ry = ry + a.y;
                    }
                }
            }
        }
    }
    if (p.initial == 0) {
        b.z = b.z + rx * (0.5f * p.dt);
        b.w = b.w + ry * (0.5f * p.dt);
    }
    accel[id] = make_float2(rx, ry);
    bodies[id] = b;
}

}  // namespace

cudaError_t launch_drift(float4* bodies, const float2* accel, int n, float half_kick, float drift_dt,
                         int substeps, GridShape g, uint32_t* keys, uint32_t* vals,
                         unsigned int* nonfinite, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    drift_kernel<<<(n + 255) / 256, 256, 0, stream>>>(bodies, accel, n, half_kick, drift_dt,
                                                      substeps, g.bounded, g.W, g.H, keys, vals,
                                                      nonfinite);
    return cudaGetLastError();
}

cudaError_t launch_kick(float4* bodies, float2* accel, const float2* force, const int* cell_start,
                        const int* cell_count, const uint32_t* cell_mass, const float4* entries,
                        KickParams p, cudaStream_t stream) {
    if (p.n <= 0) return cudaSuccess;
    kick_kernel<<<(p.n + 255) / 256, 256, 0, stream>>>(bodies, accel, force, cell_start,
                                                       cell_count, cell_mass, entries, p);
    return cudaGetLastError();
}

}  // namespace p3m
