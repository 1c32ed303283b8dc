// p3m_adjoint.cu — kernels of the reverse pass through one gravity-only step.
//
// The forward step (drift, lists, mesh force, short range, kick; the path of
// GravityPipeline.kt:445-494 without collisions) maps (x, v, a) to
//   v_h = v + a dt/2,  x' = x + v_h dt,  a' = F(x'),  v' = v_h + a' dt/2
// and its reverse maps the cotangents (lx', lv', la') to
//   wa = la' + lv' dt/2                     (cotangent of a' = F(x'))
//   lx = lx' + (dF/dx')^T wa
//   lv = lv' + lx dt,  la = lv dt/2.
// F is differentiated with the cell topology of x' held fixed (which cells
// act as monopoles and which list entries are summed is piecewise constant
// in the positions) and with the fixed-point deposit taken as its real
// value. (dF/dx)^T wa has four parts:
//   1. the mesh force interpolated with CIC weights w_i(c) (kick.comp:82-103):
//      the weights' gradient against wa_i . E(c);
//   2. the deposit (build_grid.comp): the spread Lambda(c) = sum_i w_i(c) wa_i
//      goes through the transposed mesh operator (p3m_fft.cu), giving mu(c),
//      and body j receives m_j times the weights' gradient against mu;
//   3. short-range pairs (kick.comp:66-80): the target moves against the
//      separation d and an exact source with it;
//   4. monopoles: the target only (the cell centre does not move).
// Parts 1 and 2 are one gather per body (adj_gather_kernel), part 2's spread
// is adj_spread_kernel, parts 3-4 adj_short_range_kernel; the last adds the
// sources' shares with float atomics, so the reverse pass is not bit
// reproducible run to run (the forward is).

#include "p3m_internal.cuh"

namespace p3m {
namespace {

struct Cic {
    int x0, x1, y0, y1;
    float tx, ty;
};

// The CIC cell and weights of kick.comp:82-103 / build_grid.comp.
__device__ __forceinline__ Cic cic_at(float px, float py, const AdjointParams& p) {
    const float gx = px * (float)p.W - 0.5f, gy = py * (float)p.H - 0.5f;
    const float flx = floorf(gx), fly = floorf(gy);
    const int bx = guard_coord(float_to_int(flx), p.MW), by = guard_coord(float_to_int(fly), p.MH);
    Cic c;
    c.tx = gx - flx;
    c.ty = gy - fly;
    c.x0 = wrap_index(bx, p.MW);
    c.x1 = wrap_index(bx + 1, p.MW);
    c.y0 = wrap_index(by, p.MH);
    c.y1 = wrap_index(by + 1, p.MH);
    return c;
}

__global__ void __launch_bounds__(256) adj_spread_kernel(const float4* __restrict__ bodies,
                                                         const float4* __restrict__ lam,
                                                         const float2* __restrict__ lam_a,
                                                         float2* __restrict__ wa,
                                                         float* __restrict__ cotangent,
                                                         AdjointParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const float4 l = lam[i];
    const float2 la = lam_a[i];
    const float2 w = make_float2(fmaf(p.cv, l.z, la.x), fmaf(p.cv, l.w, la.y));
    wa[i] = w;
    if (!p.mutual) return;
    const float4 b = bodies[i];
    const Cic c = cic_at(b.x, b.y, p);
    const float w00 = (1.0f - c.tx) * (1.0f - c.ty), w10 = c.tx * (1.0f - c.ty);
    const float w01 = (1.0f - c.tx) * c.ty, w11 = c.tx * c.ty;
    // Row 2y holds the x component of row y, row 2y+1 the y component.
    float* r0x = cotangent + (size_t)(2 * c.y0) * p.MW;
    float* r0y = r0x + p.MW;
    float* r1x = cotangent + (size_t)(2 * c.y1) * p.MW;
    float* r1y = r1x + p.MW;
    atomicAdd(r0x + c.x0, w00 * w.x);
    atomicAdd(r0y + c.x0, w00 * w.y);
    atomicAdd(r0x + c.x1, w10 * w.x);
    atomicAdd(r0y + c.x1, w10 * w.y);
    atomicAdd(r1x + c.x0, w01 * w.x);
    atomicAdd(r1y + c.x0, w01 * w.y);
    atomicAdd(r1x + c.x1, w11 * w.x);
    atomicAdd(r1y + c.x1, w11 * w.y);
}

struct PairK {
    float aspect, aspect2x2, inv_2s2, neg_log2e_over_2s2, min_dist2, g_over_m;
};

// J^T w for the pair term a = G m exp(-r^2/2s^2) d / (M max(r^2, r_min^2)),
// d = source - target (unit coordinates, x scaled by the aspect in r).
__device__ __forceinline__ float2 pair_vjp(const PairK& k, float dx, float dy, float m,
                                           float2 w) {
    const float px = dx * k.aspect;
    const float r2 = fmaf(px, px, dy * dy);
    const float e = exp2f(r2 * k.neg_log2e_over_2s2);
    const float phys = k.g_over_m * m * e / fmaxf(r2, k.min_dist2);
    float dphys = -phys * k.inv_2s2;
    if (r2 > k.min_dist2) dphys -= phys / r2;
    const float wd = fmaf(w.x, dx, w.y * dy);
    const float s = 2.0f * dphys * wd;
    return make_float2(fmaf(phys, w.x, s * k.aspect * k.aspect * dx), fmaf(phys, w.y, s * dy));
}

__global__ void __launch_bounds__(256) adj_short_range_kernel(
    const float4* __restrict__ bodies, const float4* __restrict__ entries,
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const uint32_t* __restrict__ cell_mass, const float2* __restrict__ wa,
    float2* __restrict__ g_short, AdjointParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const float2 w = wa[i];
    if (w.x == 0.0f && w.y == 0.0f) return;  // every term is a multiple of w
    const float4 t = bodies[i];
    PairK k;
    k.aspect = p.aspect;
    const float sigma = p.sigma_cells / (float)p.H;
    k.inv_2s2 = 1.0f / (2.0f * sigma * sigma);
    k.neg_log2e_over_2s2 = -1.4426950408889634f * k.inv_2s2;
    const float cw = p.aspect / (float)p.W, ch = 1.0f / (float)p.H;
    const float md = p.min_frac * fminf(cw, ch);
    k.min_dist2 = md * md;
    k.g_over_m = p.gravity / p.total_mass;
    const float inv_w = 1.0f / (float)p.W, inv_h = 1.0f / (float)p.H;
    const int hx = guard_coord(float_to_int(floorf(t.x * (float)p.W)), p.W);
    const int hy = guard_coord(float_to_int(floorf(t.y * (float)p.H)), p.H);
    float gx = 0.0f, gy = 0.0f;
    for (int b = -p.ry; b <= p.ry; ++b) {
        const int cy = hy + b;
        if (p.bounded && (cy < 0 || cy >= p.H)) continue;
        const int wy = wrap_index(cy, p.H);
        const float shift_y = (float)(cy - wy) * inv_h;
        for (int a = -p.rx; a <= p.rx; ++a) {
            const int cx = hx + a;
            if (p.bounded && (cx < 0 || cx >= p.W)) continue;
            const int wx = wrap_index(cx, p.W);
            const float shift_x = (float)(cx - wx) * inv_w;
            const int index = wy * p.W + wx;
            const int count = __ldg(&cell_count[index]);
            if (count == 0) continue;
            const bool home = a == 0 && b == 0;
            if (!home && count > p.exact) {
                const float mass = (float)__ldg(&cell_mass[index]) * (1.0f / kCellMassUnits);
                const float dx = ((float)wx + 0.5f) * inv_w + shift_x - t.x;
                const float dy = ((float)wy + 0.5f) * inv_h + shift_y - t.y;
                const float2 j = pair_vjp(k, dx, dy, mass, w);
                gx -= j.x;
                gy -= j.y;
            } else {
                const int limit = home ? p.home_limit : p.exact;
                const int walk = count < limit ? count : limit;
                const int start = __ldg(&cell_start[index]);
                for (int e = 0; e < walk; ++e) {
                    const float4 o = __ldg(&entries[start + e]);
                    const uint32_t src = __float_as_uint(o.w);
                    if (src == (uint32_t)i || src >= (uint32_t)p.n) continue;
                    const float2 j = pair_vjp(k, (o.x + shift_x) - t.x, (o.y + shift_y) - t.y, o.z, w);
                    gx -= j.x;
                    gy -= j.y;
                    atomicAdd(&g_short[src].x, j.x);
                    atomicAdd(&g_short[src].y, j.y);
                }
            }
        }
    }
    atomicAdd(&g_short[i].x, gx);
    atomicAdd(&g_short[i].y, gy);
}

__global__ void __launch_bounds__(256) adj_gather_kernel(
    const float4* __restrict__ bodies, const float4* __restrict__ materials,
    const float2* __restrict__ wa, const float2* __restrict__ mu2,
    const float2* __restrict__ force, const float2* __restrict__ g_short,
    float4* __restrict__ lam, float2* __restrict__ lam_a, AdjointParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float4 l = lam[i];
    if (p.mutual) {
        const float4 b = bodies[i];
        const float m = materials[i].x;
        const float2 w = wa[i];
        const Cic c = cic_at(b.x, b.y, p);
        // mu(x, y) is component (y & 1) of mu2[(y >> 1) * MW + x].
        auto phi = [&](int x, int y) {
            const float2 q = __ldg(&mu2[(size_t)(y >> 1) * p.MW + x]);
            const float2 e = __ldg(&force[(size_t)y * p.MW + x]);
            const float mu = (y & 1) ? q.y : q.x;
            return fmaf(m, mu, fmaf(w.x, e.x, w.y * e.y));
        };
        const float f00 = phi(c.x0, c.y0), f10 = phi(c.x1, c.y0);
        const float f01 = phi(c.x0, c.y1), f11 = phi(c.x1, c.y1);
        const float2 s = g_short[i];
        l.x += (float)p.W * ((f10 - f00) * (1.0f - c.ty) + (f11 - f01) * c.ty) + s.x;
        l.y += (float)p.H * ((f01 - f00) * (1.0f - c.tx) + (f11 - f10) * c.tx) + s.y;
    }
    if (p.fold) {
        lam_a[i] = make_float2(0.0f, 0.0f);
    } else {
        l.z = fmaf(p.dt, l.x, l.z);
        l.w = fmaf(p.dt, l.y, l.w);
        lam_a[i] = make_float2(0.5f * p.dt * l.z, 0.5f * p.dt * l.w);
    }
    lam[i] = l;
}

}  // namespace

cudaError_t launch_adjoint_spread(const float4* bodies, const float4* lam, const float2* lam_a,
                                  float2* wa, float* cotangent, const AdjointParams& p,
                                  cudaStream_t stream) {
    if (p.n <= 0) return cudaSuccess;
    adj_spread_kernel<<<(p.n + 255) / 256, 256, 0, stream>>>(bodies, lam, lam_a, wa, cotangent, p);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_short_range(const float4* bodies, const float4* entries,
                                       const int* cell_start, const int* cell_count,
                                       const uint32_t* cell_mass, const float2* wa,
                                       float2* g_short, const AdjointParams& p,
                                       cudaStream_t stream) {
    if (p.n <= 0 || !p.mutual) return cudaSuccess;
    adj_short_range_kernel<<<(p.n + 127) / 128, 128, 0, stream>>>(
        bodies, entries, cell_start, cell_count, cell_mass, wa, g_short, p);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_gather(const float4* bodies, const float4* materials, const float2* wa,
                                  const float2* mu2, const float2* force, const float2* g_short,
                                  float4* lam, float2* lam_a, const AdjointParams& p,
                                  cudaStream_t stream) {
    if (p.n <= 0) return cudaSuccess;
    adj_gather_kernel<<<(p.n + 255) / 256, 256, 0, stream>>>(bodies, materials, wa, mu2, force,
                                                             g_short, lam, lam_a, p);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace p3m
