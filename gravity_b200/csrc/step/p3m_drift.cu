// p3m_drift.cu — the leapfrog drift of the gravity step.
//
// Every multiply and add rounds on its own (explicit round-to-nearest
// intrinsics, never contracted into one multiply-add), as in the oracle, so
// positions and the cell keys derived from them are bit-identical to it for
// the same accelerations.
//
// drift: collision_build.comp:40-51 (gravity-only, so only the half kick,
//   drift and wall clamp / torus wrap of each collision substep), all S
//   substeps in registers, then the home-cell key of the cell sort.

#include "p3m_internal.cuh"

namespace p3m {
namespace {

// floorf(v) without the conversion unit (the drift's 32 floors per body
// otherwise saturate it): for |v| < 2^23 the round-down sum v + 2^23 (with
// v's sign) has a unit in the last place of 1, so subtracting 2^23 again
// leaves floor(v) exactly; copysign restores floorf's signed zero. Larger
// |v|, infinities and NaN are their own floor.
__device__ __forceinline__ float floor_exact(float v) {
    const float m = copysignf(8388608.0f, v);
    const float f = copysignf(__fsub_rn(__fadd_rd(v, m), m), v);
    return fabsf(v) < 8388608.0f ? f : v;
}

__device__ __forceinline__ float fractf(float v) { return __fsub_rn(v, floor_exact(v)); }

// Drifts body `id` (when id < n) and writes its cell key; returns the key.
__device__ __forceinline__ uint32_t drift_one(int id, float4* __restrict__ bodies,
                                              const float2* __restrict__ accel, int n,
                                              float half_kick, float drift_dt, int substeps,
                                              int bounded, int W, int H,
                                              uint32_t* __restrict__ keys,
                                              uint32_t* __restrict__ vals,
                                              unsigned int* __restrict__ nonfinite) {
    if (id >= n) return 0u;
    float4 b = bodies[id];
    const float2 a = accel[id];
    for (int s = 0; s < substeps; ++s) {
        // Substeps after the first carry kickDt = 0 (GravityPipeline.kt:465-473),
        // whose kick adds a * 0.
        const float hk = s == 0 ? half_kick : 0.0f;
        b.z = __fadd_rn(b.z, __fmul_rn(a.x, hk));
        b.w = __fadd_rn(b.w, __fmul_rn(a.y, hk));
        b.x = __fadd_rn(b.x, __fmul_rn(b.z, drift_dt));
        b.y = __fadd_rn(b.y, __fmul_rn(b.w, drift_dt));
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
    uint32_t key = 0u;
    if (keys) {
        const int hx = wrap_index(float_to_int(floorf(b.x * (float)W)), W);
        const int hy = wrap_index(float_to_int(floorf(b.y * (float)H)), H);
        const int slot = n - 1 - id;  // descending ID order for the cell sort
        key = (uint32_t)hx + (uint32_t)hy * (uint32_t)W;
        keys[slot] = key;
        vals[slot] = (uint32_t)id;
    }
    return key;
}

__device__ __forceinline__ void drift_body(int block, float4* __restrict__ bodies,
                                           const float2* __restrict__ accel, int n,
                                           float half_kick, float drift_dt, int substeps,
                                           int bounded, int W, int H, uint32_t* __restrict__ keys,
                                           uint32_t* __restrict__ vals,
                                           unsigned int* __restrict__ nonfinite) {
    drift_one(block * blockDim.x + threadIdx.x, bodies, accel, n, half_kick, drift_dt, substeps,
              bounded, W, H, keys, vals, nonfinite);
}

// The drift, and (totals.totals set) the digit totals of the cell keys for
// the look-back sort that follows.
__global__ void drift_kernel(float4* __restrict__ bodies, const float2* __restrict__ accel, int n,
                             float half_kick, float drift_dt, int substeps, int bounded, int W,
                             int H, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                             unsigned int* __restrict__ nonfinite, SortTotals totals) {
    grid_dependency_wait();
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t key = drift_one(id, bodies, accel, n, half_kick, drift_dt, substeps, bounded,
                                   W, H, keys, vals, nonfinite);
    if (totals.totals && keys) {
        __shared__ uint32_t sh[kSortMaxPasses * kLookbackMaxRadix];
        add_digit_totals(totals, id < n, key, sh);
    }
}

__global__ void drift_batched_kernel(const DriftArgs* __restrict__ args, const int* __restrict__ first,
                                     int sims) {
    const int2 sb = batch_block(first, sims);
    const DriftArgs a = args[sb.x];
    drift_body(sb.y, a.bodies, a.accel, a.n, a.half_kick, a.drift_dt, a.substeps, a.bounded, a.W,
               a.H, a.keys, a.vals, a.nonfinite);
}

}  // namespace

// Host-side launchers: not part of the coherent copy of the bodies that the
// batched form's persistent kernel uses (p3m_step.cu).
#ifndef P3M_COHERENT_BODIES

cudaError_t batched_drift(const DriftArgs* a, BatchGrid g, cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    drift_batched_kernel<<<g.blocks, kBatchThreads, 0, s>>>(a, g.first, g.sims);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_drift(float4* bodies, const float2* accel, int n, float half_kick, float drift_dt,
                         int substeps, GridShape g, uint32_t* keys, uint32_t* vals,
                         unsigned int* nonfinite, cudaStream_t stream, SortTotals totals) {
    if (n <= 0) return cudaSuccess;
    launch_chained(drift_kernel, (n + 255) / 256, 256, 0, stream, bodies, accel, n, half_kick,
                   drift_dt, substeps, g.bounded, g.W, g.H, keys, vals, nonfinite, totals);
    count_launches(1);
    return cudaGetLastError();
}

#endif  // !P3M_COHERENT_BODIES
}  // namespace p3m
