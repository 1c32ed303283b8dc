// p3m_deposit.cu — CIC mass deposit reduced in shared memory per sorted tile.
//
// Restates build_grid.comp:53-69: each body spreads mass * CIC weight over the
// four mesh cells around p * (W, H) - 0.5, as fixed-point integers, with the
// mesh wrap of wrapMesh (build_grid.comp:29-42). Integer sums commute, so the
// grid is bit-identical whatever the order of the additions.
//
// B200 layout: the bodies arrive in cell order (the `entries` of the cell
// sort), so one CTA's chunk of consecutive entries covers a contiguous range
// of home cells c0..c1. Its CIC footprint lies in the row-major mesh index
// window [(y0-1)*MW + x0-1, (y1+1)*MW + x1+1]. The CTA accumulates that window
// in shared memory with shared atomics and flushes each non-zero cell once with
// a global atomic. Deposits that wrap across the mesh edge, or that fall
// beyond the window's shared-memory capacity, go straight to global memory.
//
// Arithmetic is written with explicit round-to-nearest intrinsics so that no
// multiply-add is contracted: the weights must round exactly as the oracle's.

#include "p3m_internal.cuh"

namespace p3m {
namespace {

constexpr int kDepositThreads = 256;
constexpr int kDepositChunk = 2048;          // entries per CTA
constexpr int kDepositWindowBytes = 96 * 1024;

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

template <typename T>
__global__ void __launch_bounds__(kDepositThreads) deposit_kernel(
    const float4* __restrict__ entries, const uint32_t* __restrict__ keys, int n, int W, int H,
    int MW, int MH, float scale, T* __restrict__ density, int window_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* window = reinterpret_cast<T*>(smem_raw);
    __shared__ long long s_lo;
    __shared__ int s_len;

    const int base = blockIdx.x * kDepositChunk;
    const int count = min(kDepositChunk, n - base);
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

}  // namespace

cudaError_t configure_deposit() {
    cudaError_t e = cudaFuncSetAttribute(deposit_kernel<unsigned long long>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kDepositWindowBytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(deposit_kernel<uint32_t>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kDepositWindowBytes);
}

cudaError_t launch_deposit(const float4* entries, const uint32_t* keys, int n, GridShape g,
                           int deposit_mode, float mass_scale, void* density,
                           cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int blocks = (n + kDepositChunk - 1) / kDepositChunk;
    if (deposit_mode == P3M_DEPOSIT_I64) {
        using T = unsigned long long;
        const int cap = kDepositWindowBytes / (int)sizeof(T);
        deposit_kernel<T><<<blocks, kDepositThreads, kDepositWindowBytes, stream>>>(
            entries, keys, n, g.W, g.H, g.MW, g.MH, 4294967296.0f, static_cast<T*>(density), cap);
    } else {
        using T = uint32_t;
        const int cap = kDepositWindowBytes / (int)sizeof(T);
        deposit_kernel<T><<<blocks, kDepositThreads, kDepositWindowBytes, stream>>>(
            entries, keys, n, g.W, g.H, g.MW, g.MH, mass_scale, static_cast<T*>(density), cap);
    }
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace p3m
