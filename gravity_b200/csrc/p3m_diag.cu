// p3m_diag.cu — FP64 diagnostics: direct-sum accelerations of a subsample of
// targets, and momentum / kinetic energy / centre-of-mass reductions.
//
// The direct sum is the law the P3M split approximates: kernel_init.comp's
// long-range kernel -G(1-exp(-r^2/2s^2)) d/(M r^2) plus kick.comp:66-80's
// short-range complement G m exp(-r^2/2s^2) d/(M max(r^2, r_min^2)) add up to
// G m d / (M max(r^2, r_min^2)) beyond r_min. On the torus the displacement
// is the minimum image (the mesh kernel's, kernel_init.comp:22-28); inside
// walls the sum is open.

#include "p3m_internal.cuh"

namespace p3m {
namespace {

constexpr int kDiagThreads = 256;

__device__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    __syncthreads();
    return t;  // valid in thread 0
}

__global__ void __launch_bounds__(kDiagThreads) direct_accel_kernel(
    const float4* __restrict__ bodies, const float4* __restrict__ materials, int n,
    const int* __restrict__ targets, double aspect, double gravity, double total_mass,
    double min_dist2, int bounded, double2* out) {
    __shared__ double sh[kDiagThreads / 32];
    const int id = targets[blockIdx.x];
    const float4 t = bodies[id];
    const double tx = t.x, ty = t.y;
    double ax = 0.0, ay = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        if (j == id) continue;
        const float4 s = bodies[j];
        double dx = (double)s.x - tx, dy = (double)s.y - ty;
        if (!bounded) {
            dx -= floor(dx + 0.5);
            dy -= floor(dy + 0.5);
        }
        const double px = dx * aspect, py = dy;
        const double r2 = px * px + py * py;
        const double k = gravity * (double)materials[j].x / (total_mass * fmax(r2, min_dist2));
        ax += k * px;
        ay += k * py;
    }
    ax = block_sum(ax, sh);
    ay = block_sum(ay, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = make_double2(ax / aspect, ay);
}

// Per-block partial sums of 6 quantities, reduced in a fixed order.
__global__ void __launch_bounds__(kDiagThreads) conservation_partial_kernel(
    const float4* __restrict__ bodies, const float4* __restrict__ materials, int n, double w,
    double h, double* partial) {
    __shared__ double sh[kDiagThreads / 32];
    double q[6] = {0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 b = bodies[i];
        const double m = materials[i].x;
        const double vx = b.z * w, vy = b.w * h;
        q[0] += m * vx;
        q[1] += m * vy;
        q[2] += 0.5 * m * (vx * vx + vy * vy);
        q[3] += m * b.x * w;
        q[4] += m * b.y * h;
        q[5] += m;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double s = block_sum(q[k], sh);
        if (threadIdx.x == 0) partial[blockIdx.x * 6 + k] = s;
    }
}

__global__ void conservation_final_kernel(const double* partial, int blocks, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double q[6] = {0, 0, 0, 0, 0, 0};
    for (int b = 0; b < blocks; ++b)
        for (int k = 0; k < 6; ++k) q[k] += partial[b * 6 + k];
    for (int k = 0; k < 6; ++k) out[k] = q[k];
    if (q[5] > 0.0) {
        out[3] = q[3] / q[5];
        out[4] = q[4] / q[5];
    }
}

}  // namespace

cudaError_t launch_direct_accel(const float4* bodies, const float4* materials, int n,
                                const int* targets, int n_targets, double aspect, double gravity,
                                double total_mass, double min_dist2, int bounded, double2* out,
                                cudaStream_t stream) {
    if (n_targets <= 0) return cudaSuccess;
    direct_accel_kernel<<<n_targets, kDiagThreads, 0, stream>>>(bodies, materials, n, targets,
                                                                aspect, gravity, total_mass,
                                                                min_dist2, bounded, out);
    count_launches(1);
    return cudaGetLastError();
}

int conservation_blocks() { return 296; }

cudaError_t launch_conservation(const float4* bodies, const float4* materials, int n, double w,
                                double h, double* partial, double* out, cudaStream_t stream) {
    const int blocks = conservation_blocks();
    conservation_partial_kernel<<<blocks, kDiagThreads, 0, stream>>>(bodies, materials, n, w, h,
                                                                     partial);
    conservation_final_kernel<<<1, 32, 0, stream>>>(partial, blocks, out);
    count_launches(2);
    return cudaGetLastError();
}

}  // namespace p3m
