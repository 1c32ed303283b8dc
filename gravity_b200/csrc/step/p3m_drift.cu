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

// v - floor(v) for v in [-1, 2) without the conversion unit: -floor(v) is
// 1, +0 or -1 from two compares, and v + (-floor(v)) is the same single
// rounding as v - floor(v) (for v = -0 both give +0).
__device__ __forceinline__ float fract_near(float v) {
    const float neg_floor = __fsub_rn((float)(v < 0.0f), (float)(v >= 1.0f));
    return __fadd_rn(v, neg_floor);
}

__device__ __forceinline__ float fract_any(float v) { return __fsub_rn(v, floorf(v)); }

// Drifts body `id` (when id < n) and writes its cell key; returns the key.
//
// Substep 0 kicks by a*dt/2, every later substep by a*0 (kickDt = 0,
// GravityPipeline.kt:465-473). Adding the same a*0 (a signed zero, or NaN
// for a non-finite a) a second time changes nothing, so from substep 1 on
// the velocity, and with it the displacement v*dt/S, are the same: they are
// computed once. On the torus, when the position is in [0, 1] and the
// displacement below half a period, every later substep's sum stays in
// [-1, 2), where fract_near is exact; one axis takes it and the other the
// conversion unit's floor, so neither pipe limits the loop.
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
    if (substeps > 0) {
        b.z = __fadd_rn(b.z, __fmul_rn(a.x, half_kick));
        b.w = __fadd_rn(b.w, __fmul_rn(a.y, half_kick));
        float dx = __fmul_rn(b.z, drift_dt), dy = __fmul_rn(b.w, drift_dt);
        if (bounded) {
            b.x = fminf(fmaxf(__fadd_rn(b.x, dx), 0.0f), kMaximumUnit);
            b.y = fminf(fmaxf(__fadd_rn(b.y, dy), 0.0f), kMaximumUnit);
        } else {
            b.x = fract_any(__fadd_rn(b.x, dx));
            b.y = fract_any(__fadd_rn(b.y, dy));
        }
        if (substeps > 1) {
            b.z = __fadd_rn(b.z, __fmul_rn(a.x, 0.0f));
            b.w = __fadd_rn(b.w, __fmul_rn(a.y, 0.0f));
            dx = __fmul_rn(b.z, drift_dt);
            dy = __fmul_rn(b.w, drift_dt);
            if (bounded) {
                for (int s = 1; s < substeps; ++s) {
                    b.x = fminf(fmaxf(__fadd_rn(b.x, dx), 0.0f), kMaximumUnit);
                    b.y = fminf(fmaxf(__fadd_rn(b.y, dy), 0.0f), kMaximumUnit);
                }
            } else if (b.x >= 0.0f && b.x <= 1.0f && fabsf(dx) < 0.5f && b.y >= 0.0f &&
                       b.y <= 1.0f && fabsf(dy) < 0.5f) {
                for (int s = 1; s < substeps; ++s) {
                    b.x = fract_any(__fadd_rn(b.x, dx));
                    b.y = fract_near(__fadd_rn(b.y, dy));
                }
            } else {
                for (int s = 1; s < substeps; ++s) {
                    b.x = fract_any(__fadd_rn(b.x, dx));
                    b.y = fract_any(__fadd_rn(b.y, dy));
                }
            }
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
