// p3m_fft.cu — real 2D FFT with the Green's-function multiply fused in.
//
// Replaces fft_init.comp, fft_shared.comp (forward + two inverse complex 2D
// transforms, GravityPipeline.kt:944-972), convolve.comp and the kernel
// spectra of kernel_init.comp (GravityPipeline.kt:1341-1357).
//
// The reference transforms the real density as a full complex mesh, convolves
// with two complex kernel spectra and runs two complex inverses. Here:
//   1. forward rows: two real density rows form one complex line
//      (z = row_a + i row_b); one complex FFT gives both rows' half spectra.
//   2. columns: for each half-spectrum column kx in [0, MW/2]: forward FFT
//      along y, multiply by the Green's function with its gradient and the CIC
//      deconvolution folded in (one table, (gx, gy) per bin), inverse FFT of
//      Fx and of Fy along y.
//   3. inverse rows: fx and fy are real, so one complex inverse of
//      Z = Fx + i Fy per row gives fx in the real and fy in the imaginary part.
// This moves 3 complex line-FFTs per mesh row/column pair instead of 6.
//
// The Green's table. The force kernels Kx, Ky of kernel_init.comp are real
// and odd (the Nyquist component is zeroed for that, kernel_init.comp:37-40),
// so their spectra are purely imaginary: K^x = i*ax, K^y = i*ay. The table
// holds g = (ax, ay) * deconvolution / (MW*MH) for unit total mass, computed
// in FP64 on the device (one packed complex FFT of Kx + i*Ky) and rounded
// once to FP32; the step multiplies by 1/M_tot. The spectral multiply is then
//   F = rho^ * i*g = (-rho^.y * g, rho^.x * g).
//
// Each line FFT is a Stockham autosort transform in shared memory, radix 8
// with a final radix-4 or -2 pass, twiddles from one FP32 table of 4096 roots
// e^{-2 pi i m / 4096} (computed in FP64 on the host).

#include "p3m_internal.cuh"

#include <cmath>

namespace p3m {
namespace {

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 caddf(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csubf(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 rot(float2 a, bool inverse) {
    return inverse ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R>
__device__ __forceinline__ void dft(float2 (&v)[R], bool inverse);

template <>
__device__ __forceinline__ void dft<2>(float2 (&v)[2], bool) {
    const float2 a = v[0], b = v[1];
    v[0] = caddf(a, b);
    v[1] = csubf(a, b);
}

template <>
__device__ __forceinline__ void dft<4>(float2 (&v)[4], bool inverse) {
    const float2 s02 = caddf(v[0], v[2]), d02 = csubf(v[0], v[2]);
    const float2 s13 = caddf(v[1], v[3]), d13 = rot(csubf(v[1], v[3]), inverse);
    v[0] = caddf(s02, s13);
    v[2] = csubf(s02, s13);
    v[1] = caddf(d02, d13);
    v[3] = csubf(d02, d13);
}

template <>
__device__ __forceinline__ void dft<8>(float2 (&v)[8], bool inverse) {
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft<4>(e, inverse);
    dft<4>(o, inverse);
    const float h = 0.70710678118654752440f;
    // o[k] *= e^{-+2 pi i k / 8}
    o[1] = inverse ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                   : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    o[2] = rot(o[2], inverse);
    o[3] = inverse ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                   : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = caddf(e[k], o[k]);
        v[k + 4] = csubf(e[k], o[k]);
    }
}

// Position of point i of a line in shared memory: bits 0-3 XOR bits 4-7.
// The passes write point (j - k) * R + k + r * Ns from lane j, strides that
// would put a warp's stores on a few banks; the swizzle spreads every pass's
// reads and writes over all banks. It permutes the points of each aligned
// 256-point block (a line of 16 points or fewer is unchanged), so a line of
// L = 2^n points stays in [0, L). Every access to a line buffer goes
// through it.
__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 4) & 15); }

// One Stockham pass of radix R over `lines` lines of length L = 2^log2L (line
// pitch `pitch`), src -> dst. Ns = product of earlier radices; log2(Ns*R) <= 12.
template <int R>
__device__ __forceinline__ void stockham_pass(const float2* __restrict__ src, float2* __restrict__ dst,
                                              int log2L, int lines, int pitch, int Ns, int log_ns_r,
                                              bool inverse, const float2* __restrict__ tw,
                                              int tw_log2) {
    constexpr int kLog2R = R == 8 ? 3 : (R == 4 ? 2 : 1);
    const int log_per_line = log2L - kLog2R;
    const int per_line = 1 << log_per_line;
    const int total = lines << log_per_line;
    const int shift = tw_log2 - log_ns_r;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int line = t >> log_per_line;
        const int j = t & (per_line - 1);
        const float2* s = src + line * pitch;
        float2* d = dst + line * pitch;
        const int k = j & (Ns - 1);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 x = s[swz(j + r * per_line)];
            if (r > 0 && k > 0) {
                float2 w = tw[(k * r) << shift];
                if (inverse) w.y = -w.y;
                x = cmulf(x, w);
            }
            v[r] = x;
        }
        dft<R>(v, inverse);
        const int out = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) d[swz(out + r * Ns)] = v[r];
    }
}

// Complex FFT of `lines` lines held in buffer a (ping-pong buffer b); returns
// the buffer that holds the result. Ends with __syncthreads(). `tw` holds the
// roots e^{-2 pi i m / 2^tw_log2}: the global 4096-root table (tw_log2 = 12)
// or a CTA's copy of the L roots its lines use (tw_log2 = log2 L).
__device__ float2* line_fft(float2* a, float2* b, int L, int log2L, int lines, int pitch,
                            bool inverse, const float2* __restrict__ tw,
                            int tw_log2 = kTwiddleLog2) {
    int Ns = 1, logNs = 0;
    while (Ns < L) {
        const int remaining = log2L - logNs;
        if (remaining >= 3) {
            stockham_pass<8>(a, b, log2L, lines, pitch, Ns, logNs + 3, inverse, tw, tw_log2);
            Ns <<= 3; logNs += 3;
        } else if (remaining == 2) {
            stockham_pass<4>(a, b, log2L, lines, pitch, Ns, logNs + 2, inverse, tw, tw_log2);
            Ns <<= 2; logNs += 2;
        } else {
            stockham_pass<2>(a, b, log2L, lines, pitch, Ns, logNs + 1, inverse, tw, tw_log2);
            Ns <<= 1; logNs += 1;
        }
        __syncthreads();
        float2* t = a; a = b; b = t;
    }
    return a;
}

__device__ __forceinline__ int ilog2(int v) { return 31 - __clz(v); }

// Global loads a thread issues before it uses the first of them, in the loops
// that fill shared memory: a CTA of 64 threads moving a 512-point column would
// otherwise wait out one memory latency per point.
constexpr int kLoadBatch = 8;

// Lines of up to this many points copy their roots into shared memory; the
// table of a longer line would cost a CTA per SM, more than its L1 misses.
constexpr int kStagedTwiddlesMax = 2048;
__host__ __device__ __forceinline__ int staged_twiddles(int L) {
    return L <= kStagedTwiddlesMax ? L : 0;
}

// The L roots e^{-2 pi i m / L} (L = 2^log2L) into shared memory, so that the
// passes of a line transform read their twiddles there instead of waiting on
// L1 misses to the global table. Values are the table's; a barrier must
// follow before use. Returns the table to pass to line_fft with log2 L, or
// the global table (log2 12) for lines longer than kStagedTwiddlesMax.
__device__ __forceinline__ const float2* stage_twiddles(const float2* __restrict__ tw, float2* dst,
                                                       int L, int log2L, int* tw_log2) {
    if (!staged_twiddles(L)) {
        *tw_log2 = kTwiddleLog2;
        return tw;
    }
    *tw_log2 = log2L;
    const int shift = kTwiddleLog2 - log2L;
    for (int m0 = threadIdx.x; m0 < L; m0 += kLoadBatch * blockDim.x) {
        float2 v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int m = m0 + u * blockDim.x;
            if (m < L) v[u] = __ldg(&tw[m << shift]);
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int m = m0 + u * blockDim.x;
            if (m < L) dst[m] = v[u];
        }
    }
    return dst;
}

// ---------------------------------------------------------------- kernels
// 1. forward rows: fft_init.comp (fixed point -> float) fused with the row
// transform. Two rows per complex line.
template <typename T>
__device__ __forceinline__ void fft_rows_forward_body(int block, const T* __restrict__ density,
                                                      float inv_scale, int MW, int MH,
                                                      int pairs_per_cta,
                                                      const float2* __restrict__ tw,
                                                      float2* __restrict__ half) {
    extern __shared__ __align__(16) float2 sm[];
    const int pair0 = block * pairs_per_cta;
    const int pairs = min(pairs_per_cta, MH / 2 - pair0);
    float2* a = sm;
    float2* b = sm + pairs_per_cta * MW;
    int twl;
    const int logW = ilog2(MW);
    const float2* tws = stage_twiddles(tw, sm + 2 * pairs_per_cta * MW, MW, logW, &twl);
    const int total = pairs * MW;
    for (int t0 = threadIdx.x; t0 < total; t0 += kLoadBatch * blockDim.x) {
        T lo[kLoadBatch], hi[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) {
                const int p = t >> logW, x = t & (MW - 1);
                const size_t row = (size_t)(pair0 + p) * 2;
                lo[u] = density[row * MW + x];
                hi[u] = density[(row + 1) * MW + x];
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) {
                const int p = t >> logW, x = t & (MW - 1);
                a[p * MW + swz(x)] = make_float2((float)lo[u] * inv_scale, (float)hi[u] * inv_scale);
            }
        }
    }
    __syncthreads();
    float2* z = line_fft(a, b, MW, logW, pairs, MW, false, tws, twl);
    const int SW = MW / 2 + 1;
    for (int p = 0; p < pairs; ++p) {
        const size_t row = (size_t)(pair0 + p) * 2;
        for (int kx = threadIdx.x; kx < SW; kx += blockDim.x) {
            const float2 zk = z[p * MW + swz(kx)];
            const float2 zn = z[p * MW + swz((MW - kx) & (MW - 1))];
            const float2 A = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
            const float2 B = make_float2(0.5f * (zk.y + zn.y), 0.5f * (zn.x - zk.x));
            half[row * SW + kx] = A;
            half[(row + 1) * SW + kx] = B;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) fft_rows_forward_kernel(const T* __restrict__ density,
                                                               float inv_scale, int MW, int MH,
                                                               int pairs_per_cta,
                                                               const float2* __restrict__ tw,
                                                               float2* __restrict__ half) {
    grid_dependency_wait();
    fft_rows_forward_body<T>(blockIdx.x, density, inv_scale, MW, MH, pairs_per_cta, tw, half);
}

template <typename T>
__global__ void __launch_bounds__(256) fft_rows_forward_batched_kernel(
    const FftRowsArgs* __restrict__ args, const int* __restrict__ first, int sims,
    const float2* __restrict__ tw) {
    const int2 sb = batch_block(first, sims);
    const FftRowsArgs a = args[sb.x];
    fft_rows_forward_body<T>(sb.y, static_cast<const T*>(a.density), a.inv_scale, a.MW, a.MH,
                             a.per_cta, tw, a.half);
}

// 2. columns: forward along y, Green's multiply (convolve.comp), inverse of Fx
// and Fy along y. Shared memory: [A: G lines | B: G lines | C: 2G lines].
__device__ __forceinline__ void fft_columns_body(int block, const float2* __restrict__ half,
                                                 const float2* __restrict__ green, float inv_total,
                                                 int MW, int MH, int G,
                                                 const float2* __restrict__ tw,
                                                 float4* __restrict__ cols) {
    extern __shared__ __align__(16) float2 sm[];
    const int SW = MW / 2 + 1;
    const int kx0 = block * G;
    const int ncols = min(G, SW - kx0);
    const int logH = ilog2(MH);
    float2* A = sm;
    float2* B = sm + G * MH;
    float2* C = sm + 2 * G * MH;
    int twl;
    const float2* tws = stage_twiddles(tw, sm + 4 * G * MH, MH, logH, &twl);
    const int total = ncols * MH;
    for (int t0 = threadIdx.x; t0 < total; t0 += kLoadBatch * blockDim.x) {
        float2 v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) {
                const int c = t >> logH, y = t & (MH - 1);
                v[u] = half[(size_t)y * SW + kx0 + c];
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) {
                const int c = t >> logH, y = t & (MH - 1);
                A[c * MH + swz(y)] = v[u];
            }
        }
    }
    // The Green's table entries of the block's bins, fetched while the
    // forward transform runs.
    float2 gv[kLoadBatch];
    const bool g_fits = total <= kLoadBatch * (int)blockDim.x;
    if (g_fits) {
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = threadIdx.x + u * blockDim.x;
            if (t < total) {
                const int c = t >> logH, y = t & (MH - 1);
                gv[u] = __ldg(&green[(size_t)y * SW + kx0 + c]);
            }
        }
    }
    __syncthreads();
    const float2* R = line_fft(A, B, MH, logH, ncols, MH, false, tws, twl);
    for (int t0 = threadIdx.x; t0 < total; t0 += kLoadBatch * blockDim.x) {
        if (!g_fits) {
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u) {
                const int t = t0 + u * blockDim.x;
                if (t < total) {
                    const int c = t >> logH, y = t & (MH - 1);
                    gv[u] = __ldg(&green[(size_t)y * SW + kx0 + c]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) {
                const int c = t >> logH, y = t & (MH - 1);
                const float2 rho = R[c * MH + swz(y)];
                const float gx = gv[u].x * inv_total, gy = gv[u].y * inv_total;
                C[c * MH + swz(y)] = make_float2(-rho.y * gx, rho.x * gx);
                C[(ncols + c) * MH + swz(y)] = make_float2(-rho.y * gy, rho.x * gy);
            }
        }
    }
    __syncthreads();
    const float2* F = line_fft(C, A, MH, logH, 2 * ncols, MH, true, tws, twl);
    for (int t = threadIdx.x; t < ncols * MH; t += blockDim.x) {
        const int c = t >> logH, y = t & (MH - 1);
        const float2 fx = F[c * MH + swz(y)], fy = F[(ncols + c) * MH + swz(y)];
        cols[(size_t)y * SW + kx0 + c] = make_float4(fx.x, fx.y, fy.x, fy.y);
    }
}

__global__ void __launch_bounds__(256) fft_columns_kernel(const float2* __restrict__ half,
                                                          const float2* __restrict__ green,
                                                          float inv_total, int MW, int MH, int G,
                                                          const float2* __restrict__ tw,
                                                          float4* __restrict__ cols) {
    grid_dependency_wait();
    fft_columns_body(blockIdx.x, half, green, inv_total, MW, MH, G, tw, cols);
}

__global__ void __launch_bounds__(256) fft_columns_batched_kernel(
    const FftColumnsArgs* __restrict__ args, const int* __restrict__ first, int sims,
    const float2* __restrict__ tw) {
    const int2 sb = batch_block(first, sims);
    const FftColumnsArgs a = args[sb.x];
    fft_columns_body(sb.y, a.half, a.green, a.inv_total, a.MW, a.MH, a.per_cta, tw, a.cols);
}

// 2'. columns of the adjoint (transposed) mesh operator. `half` holds the
// row spectra of the two cotangent fields interleaved by row (row 2y: X, row
// 2y+1: Y, as fft_rows_forward_kernel leaves a field of 2*MH rows). Each
// column of X and Y is transformed along y, combined as
//   mu^ = Kx^T X^ + Ky^T Y^ = -(i gx X^ + i gy Y^) / M
// (the gradient kernels are real and odd, so each transpose is the negated
// operator), and transformed back; row y of mu^ goes to component (y & 1) of
// the complex pair at cols[(y >> 1) * SW + kx], the layout
// fft_rows_inverse_kernel turns into two real rows per float2.
__global__ void __launch_bounds__(256) fft_columns_adjoint_kernel(const float2* __restrict__ half,
                                                                  const float2* __restrict__ green,
                                                                  float inv_total, int MW, int MH,
                                                                  int G,
                                                                  const float2* __restrict__ tw,
                                                                  float2* __restrict__ cols) {
    extern __shared__ __align__(16) float2 sm[];
    const int SW = MW / 2 + 1;
    const int kx0 = blockIdx.x * G;
    const int ncols = min(G, SW - kx0);
    const int logH = ilog2(MH);
    float2* A = sm;               // 2G lines: X columns, then Y columns
    float2* B = sm + 2 * G * MH;  // 2G lines
    int twl;
    const float2* tws = stage_twiddles(tw, sm + 4 * G * MH, MH, logH, &twl);
    // Line l = comp * ncols + c holds component comp of column c; a thread
    // takes points of one line at a time (shifts, no division).
    const int total2 = 2 * ncols * MH;
    for (int t0 = threadIdx.x; t0 < total2; t0 += kLoadBatch * blockDim.x) {
        float2 v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total2) {
                const int l = t >> logH, y = t & (MH - 1);
                const int comp = l >= ncols ? 1 : 0, c = l - comp * ncols;
                v[u] = half[(size_t)(2 * y + comp) * SW + kx0 + c];
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total2) A[(t >> logH) * MH + swz(t & (MH - 1))] = v[u];
        }
    }
    __syncthreads();
    float2* R = line_fft(A, B, MH, logH, 2 * ncols, MH, false, tws, twl);
    float2* C = R == A ? B : A;
    const int total = ncols * MH;
    for (int t0 = threadIdx.x; t0 < total; t0 += kLoadBatch * blockDim.x) {
        float2 gv[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) {
                const int c = t >> logH, y = t & (MH - 1);
                gv[u] = __ldg(&green[(size_t)y * SW + kx0 + c]);
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) {
                const int c = t >> logH, y = t & (MH - 1);
                const float2 X = R[c * MH + swz(y)], Y = R[(ncols + c) * MH + swz(y)];
                const float2 g = gv[u];
                const float sx = X.x * g.x + Y.x * g.y, sy = X.y * g.x + Y.y * g.y;
                C[c * MH + swz(y)] = make_float2(sy * inv_total, -sx * inv_total);  // -i (gx X + gy Y) / M
            }
        }
    }
    __syncthreads();
    const float2* F = line_fft(C, R, MH, logH, ncols, MH, true, tws, twl);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int c = t >> logH, y = t & (MH - 1);
        cols[((size_t)(y >> 1) * SW + kx0 + c) * 2 + (y & 1)] = F[c * MH + swz(y)];
    }
}

// Forward column transform only (the density spectrum, for diagnostics).
__global__ void __launch_bounds__(256) fft_columns_forward_kernel(float2* half, int MW, int MH,
                                                                  int G,
                                                                  const float2* __restrict__ tw) {
    extern __shared__ __align__(16) float2 sm[];
    const int SW = MW / 2 + 1;
    const int kx0 = blockIdx.x * G;
    const int ncols = min(G, SW - kx0);
    float2* A = sm;
    float2* B = sm + G * MH;
    for (int t = threadIdx.x; t < ncols * MH; t += blockDim.x) {
        const int y = t / ncols, c = t - y * ncols;
        A[c * MH + swz(y)] = half[(size_t)y * SW + kx0 + c];
    }
    __syncthreads();
    const float2* R = line_fft(A, B, MH, ilog2(MH), ncols, MH, false, tw);
    for (int t = threadIdx.x; t < ncols * MH; t += blockDim.x) {
        const int y = t / ncols, c = t - y * ncols;
        half[(size_t)y * SW + kx0 + c] = R[c * MH + swz(y)];
    }
}

// 3. inverse rows: Z = Fx + i Fy over the full row from the two half spectra
// (each Hermitian in kx), one complex inverse, (fx, fy) = (Re, Im).
__device__ __forceinline__ void fft_rows_inverse_body(int block, const float4* __restrict__ cols,
                                                      int MW, int MH, int rows_per_cta,
                                                      const float2* __restrict__ tw,
                                                      float2* __restrict__ force) {
    extern __shared__ __align__(16) float2 sm[];
    const int row0 = block * rows_per_cta;
    const int rows = min(rows_per_cta, MH - row0);
    const int SW = MW / 2 + 1;
    float2* a = sm;
    float2* b = sm + rows_per_cta * MW;
    int twl;
    const float2* tws = stage_twiddles(tw, sm + 2 * rows_per_cta * MW, MW, ilog2(MW), &twl);
    for (int r = 0; r < rows; ++r) {
        for (int k0 = threadIdx.x; k0 < SW; k0 += kLoadBatch * blockDim.x) {
            float4 v[kLoadBatch];
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u) {
                const int kx = k0 + u * blockDim.x;
                if (kx < SW) v[u] = cols[(size_t)(row0 + r) * SW + kx];  // (Fx.re, Fx.im, Fy.re, Fy.im)
            }
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u) {
                const int kx = k0 + u * blockDim.x;
                if (kx < SW) {
                    const float4 q = v[u];
                    if (kx == 0 || kx == MW / 2) {
                        // DC and Nyquist bins of a real row are real.
                        a[r * MW + swz(kx)] = make_float2(q.x, q.z);
                    } else {
                        a[r * MW + swz(kx)] = make_float2(q.x - q.w, q.y + q.z);
                        a[r * MW + swz(MW - kx)] = make_float2(q.x + q.w, q.z - q.y);
                    }
                }
            }
        }
    }
    __syncthreads();
    const int logW = ilog2(MW);
    const float2* z = line_fft(a, b, MW, logW, rows, MW, true, tws, twl);
    for (int t = threadIdx.x; t < rows * MW; t += blockDim.x) {
        const int r = t >> logW, x = t & (MW - 1);
        force[(size_t)(row0 + r) * MW + x] = z[r * MW + swz(x)];
    }
}

__global__ void __launch_bounds__(256) fft_rows_inverse_kernel(const float4* __restrict__ cols,
                                                               int MW, int MH, int rows_per_cta,
                                                               const float2* __restrict__ tw,
                                                               float2* __restrict__ force) {
    grid_dependency_wait();
    fft_rows_inverse_body(blockIdx.x, cols, MW, MH, rows_per_cta, tw, force);
}

__global__ void __launch_bounds__(256) fft_rows_inverse_batched_kernel(
    const FftInverseArgs* __restrict__ args, const int* __restrict__ first, int sims,
    const float2* __restrict__ tw) {
    const int2 sb = batch_block(first, sims);
    const FftInverseArgs a = args[sb.x];
    fft_rows_inverse_body(sb.y, a.cols, a.MW, a.MH, a.per_cta, tw, a.force);
}

// ------------------------------------------------------- FP64 Green's table
// kernel_init.comp:16-46 in FP64 with unit total mass, packed as Kx + i Ky.
__global__ void green_real_kernel(double2* z, int MW, int MH, int W, int H, double aspect,
                                  double gravity, double sigma_cells) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)MW * MH) return;
    const int raw_x = (int)(id % MW), raw_y = (int)(id / MW);
    const int off_x = raw_x <= MW / 2 ? raw_x : raw_x - MW;
    const int off_y = raw_y <= MH / 2 ? raw_y : raw_y - MH;
    const double dx = (double)off_x * aspect / (double)W;
    const double dy = (double)off_y / (double)H;
    const double r2 = dx * dx + dy * dy;
    if (r2 == 0.0) {
        z[id] = make_double2(0.0, 0.0);
        return;
    }
    const double sigma = sigma_cells / (double)H;
    const double long_w = 1.0 - exp(-r2 / (2.0 * sigma * sigma));
    const double dir_x = raw_x * 2 == MW ? 0.0 : dx;
    const double dir_y = raw_y * 2 == MH ? 0.0 : dy;
    const double scale = -gravity * long_w / r2;
    z[id] = make_double2(scale * dir_x / aspect, scale * dir_y);
}

// FP64 radix-2 in-place FFT of one line per CTA (the layout of
// fft_shared.comp, exact twiddles from sincospi). axis 0 = rows, 1 = columns.
__global__ void fft64_line_kernel(double2* z, int MW, int MH, int axis) {
    extern __shared__ __align__(16) double2 ld[];
    const int L = axis == 0 ? MW : MH;
    const int bits = ilog2(L);
    const int line = blockIdx.x;
    auto gidx = [&](int c) -> size_t {
        return axis == 0 ? (size_t)line * MW + c : (size_t)c * MW + line;
    };
    for (int c = threadIdx.x; c < L; c += blockDim.x) {
        const int src = bits ? (int)(__brev((unsigned)c) >> (32 - bits)) : 0;
        ld[c] = z[gidx(src)];
    }
    __syncthreads();
    for (int stage = 2; stage <= L; stage <<= 1) {
        const int h = stage >> 1;
        for (int bf = threadIdx.x; bf < L / 2; bf += blockDim.x) {
            const int within = bf & (h - 1);
            const int lower = (bf / h) * stage + within;
            double s, c;
            sincospi(-2.0 * (double)within / (double)stage, &s, &c);
            const double2 lo = ld[lower], up = ld[lower + h];
            const double2 u = make_double2(c * up.x - s * up.y, c * up.y + s * up.x);
            ld[lower] = make_double2(lo.x + u.x, lo.y + u.y);
            ld[lower + h] = make_double2(lo.x - u.x, lo.y - u.y);
        }
        __syncthreads();
    }
    for (int c = threadIdx.x; c < L; c += blockDim.x) z[gidx(c)] = ld[c];
}

// Z = K^x + i K^y = i ax - ay, so ax = Im Z, ay = -Re Z. Deconvolution of
// convolve.comp:30-42 in FP64.
__global__ void green_final_kernel(const double2* z, int MW, int MH, double window_floor,
                                   float2* green) {
    const int SW = MW / 2 + 1;
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)SW * MH) return;
    const int kx = (int)(id % SW), ky = (int)(id / SW);
    const int ikx = kx;  // kx <= MW/2
    const int iky = ky <= MH / 2 ? ky : ky - MH;
    auto sinc = [](double v) { return fabs(v) < 1e-12 ? 1.0 : sin(v) / v; };
    const double sx = sinc(M_PI * (double)ikx / (double)MW);
    const double sy = sinc(M_PI * (double)iky / (double)MH);
    const double window = sx * sx * sy * sy;
    const double deconv = 1.0 / fmax(window * window, window_floor);
    const double scale = deconv / ((double)MW * (double)MH);
    const double2 v = z[(size_t)ky * MW + kx];
    green[id] = make_float2((float)(v.y * scale), (float)(-v.x * scale));
}

// The density mesh as FP64 complex values (count / massScale, 0): the input
// of validateFft's double-precision transform (GravityPipeline.kt:386-393).
// The integer counts convert exactly; one FP64 product follows.
__global__ void density_f64_kernel(const void* __restrict__ density, int i64, double inv_scale,
                                   long long M, double2* __restrict__ z) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= M) return;
    const double v = i64 ? (double)static_cast<const long long*>(density)[id]
                         : (double)static_cast<const uint32_t*>(density)[id];
    z[id] = make_double2(v * inv_scale, 0.0);
}

inline int ilog2_host(int v) {
    int b = 0;
    while ((1 << (b + 1)) <= v) ++b;
    return b;
}

cudaError_t set_smem(const void* fn, size_t bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Lines per CTA: enough CTAs for two per SM (296) when there are that many
// lines, at most `cap`; threads: one radix-8 butterfly per thread and pass,
// 64..256.
void line_shape(int lines_total, int L, int cap, int* per_cta, int* threads, int fixed = 0) {
    int g = fixed > 0 ? fixed : lines_total / 296;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    *per_cta = g;
    int t = ((g * L / 8) + 31) / 32 * 32;
    *threads = t < 64 ? 64 : (t > 256 ? 256 : t);
}

// Columns per CTA of the column kernels: at most 16 and at most what 64 KB
// of shared memory holds, so that three CTAs share an SM even for
// 2048-point columns (the kernels are latency-bound: at 4096x2048 one
// 128 KB CTA per SM took the spectral pass 0.18 ms, three of 64 KB 0.14).
void column_shape(int MW, int MH, int lines_factor, int* G, int* threads, int fixed) {
    const int SW = MW / 2 + 1;
    int cap = (64 * 1024) / (lines_factor * MH * (int)sizeof(float2));
    if (cap > 16) cap = 16;
    line_shape(SW, MH, cap, G, threads, fixed);
}

}  // namespace

// Host-side launchers: not part of the coherent copy of the bodies that the
// batched form's persistent kernel uses (p3m_step.cu).
#ifndef P3M_COHERENT_BODIES

// Dynamic shared memory opt-in (above 48 KB) of every FFT kernel, once per
// device at context creation (never inside a stream capture).
cudaError_t configure_fft() {
    const size_t big = 200 * 1024;
    const void* fns[] = {(const void*)fft_rows_forward_kernel<long long>,
                         (const void*)fft_rows_forward_kernel<uint32_t>,
                         (const void*)fft_rows_forward_kernel<float>,
                         (const void*)fft_columns_adjoint_kernel,
                         (const void*)fft_rows_forward_batched_kernel<long long>,
                         (const void*)fft_rows_forward_batched_kernel<uint32_t>,
                         (const void*)fft_columns_batched_kernel,
                         (const void*)fft_rows_inverse_batched_kernel,
                         (const void*)fft_columns_kernel, (const void*)fft_columns_forward_kernel,
                         (const void*)fft_rows_inverse_kernel, (const void*)fft64_line_kernel};
    for (const void* f : fns) {
        cudaError_t e = set_smem(f, big);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void host_twiddles(float2* out) {
    for (int m = 0; m < kTwiddleLength; ++m) {
        const double a = -2.0 * M_PI * (double)m / (double)kTwiddleLength;
        out[m] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
}

cudaError_t launch_fft_forward_rows(const void* density, int deposit_mode, float inv_scale,
                                    GridShape g, const float2* twiddles, float2* half,
                                    cudaStream_t stream) {
    const int pairs = g.MH / 2;
    int pairs_per_cta, threads;
    line_shape(pairs, g.MW, g.MW >= 4096 ? 1 : 4096 / g.MW, &pairs_per_cta, &threads, g.fft_lines);
    const int blocks = (pairs + pairs_per_cta - 1) / pairs_per_cta;
    const size_t smem = ((size_t)2 * pairs_per_cta * g.MW + staged_twiddles(g.MW)) * sizeof(float2);
    if (deposit_mode == P3M_DEPOSIT_I64) {
        launch_chained(fft_rows_forward_kernel<long long>, blocks, threads, smem, stream,
            static_cast<const long long*>(density), inv_scale, g.MW, g.MH, pairs_per_cta, twiddles,
            half);
    } else {
        launch_chained(fft_rows_forward_kernel<uint32_t>, blocks, threads, smem, stream,
            static_cast<const uint32_t*>(density), inv_scale, g.MW, g.MH, pairs_per_cta, twiddles,
            half);
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fft_columns(const float2* half, const float2* green, float inv_total,
                               GridShape g, const float2* twiddles, float4* cols,
                               cudaStream_t stream) {
    int G, threads;
    column_shape(g.MW, g.MH, 4, &G, &threads, g.fft_lines);
    const int SW = g.MW / 2 + 1;
    const int blocks = (SW + G - 1) / G;
    const size_t smem = ((size_t)4 * G * g.MH + staged_twiddles(g.MH)) * sizeof(float2);
    launch_chained(fft_columns_kernel, blocks, threads, smem, stream, half, green, inv_total, g.MW, g.MH, G,
                                                      twiddles, cols);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fft_adjoint(const float* cotangent, const float2* green, float inv_total,
                               GridShape g, const float2* twiddles, float2* half2, float4* cols,
                               float2* mu2, cudaStream_t stream) {
    // Rows: the 2*MH-row field (X and Y rows interleaved), two rows per line.
    {
        const int pairs = g.MH;
        int pairs_per_cta, threads;
        line_shape(pairs, g.MW, g.MW >= 4096 ? 1 : 4096 / g.MW, &pairs_per_cta, &threads, g.fft_lines);
        const int blocks = (pairs + pairs_per_cta - 1) / pairs_per_cta;
        const size_t smem = ((size_t)2 * pairs_per_cta * g.MW + staged_twiddles(g.MW)) * sizeof(float2);
        fft_rows_forward_kernel<float><<<blocks, threads, smem, stream>>>(
            cotangent, 1.0f, g.MW, 2 * g.MH, pairs_per_cta, twiddles, half2);
        count_launches(1);
    }
    {
        int G, threads;
        column_shape(g.MW, g.MH, 4, &G, &threads, g.fft_lines);
        const int SW = g.MW / 2 + 1;
        const int blocks = (SW + G - 1) / G;
        const size_t smem = ((size_t)4 * G * g.MH + staged_twiddles(g.MH)) * sizeof(float2);
        fft_columns_adjoint_kernel<<<blocks, threads, smem, stream>>>(
            half2, green, inv_total, g.MW, g.MH, G, twiddles, reinterpret_cast<float2*>(cols));
        count_launches(1);
    }
    // Inverse rows: pairs of mu rows as the real and imaginary parts.
    {
        const int rows = g.MH / 2;
        int rows_per_cta, threads;
        line_shape(rows, g.MW, g.MW >= 4096 ? 1 : 4096 / g.MW, &rows_per_cta, &threads, g.fft_lines);
        const int blocks = (rows + rows_per_cta - 1) / rows_per_cta;
        const size_t smem = ((size_t)2 * rows_per_cta * g.MW + staged_twiddles(g.MW)) * sizeof(float2);
        launch_chained(fft_rows_inverse_kernel, blocks, threads, smem, stream, cols, g.MW, rows, rows_per_cta,
                                                               twiddles, mu2);
        count_launches(1);
    }
    return cudaGetLastError();
}

// Batched launches run 256 threads per CTA for every simulation: enough
// lines per CTA that one radix-8 pass gives every thread a butterfly
// (lines * L / 8 >= 256), within the shared-memory caps of the single
// launches and the simulation's line count.
void fft_batch_shape(const GridShape& g, int* rows_per_cta, int* cols_per_cta, int* inv_per_cta,
                     size_t* rows_smem, size_t* cols_smem, size_t* inv_smem) {
    // Lines per CTA: the autotuner's choice (g.fft_lines), else as many as
    // make one radix-8 pass fill 256 threads; at most `cap` and the lines.
    auto fill = [&g](int lines_total, int L, int cap) {
        int per = g.fft_lines > 0 ? g.fft_lines : (256 * 8 + L - 1) / L;
        if (per > cap) per = cap;
        if (per > lines_total) per = lines_total;
        return per < 1 ? 1 : per;
    };
    const int row_cap = g.MW >= 4096 ? 1 : 4096 / g.MW;
    int col_cap = (64 * 1024) / (4 * g.MH * (int)sizeof(float2));
    if (col_cap > 16) col_cap = 16;
    *rows_per_cta = fill(g.MH / 2, g.MW, row_cap);
    // + the staged twiddles of one line
    *rows_smem = ((size_t)2 * *rows_per_cta * g.MW + staged_twiddles(g.MW)) * sizeof(float2);
    *cols_per_cta = fill(g.MW / 2 + 1, g.MH, col_cap);
    *cols_smem = ((size_t)4 * *cols_per_cta * g.MH + staged_twiddles(g.MH)) * sizeof(float2);
    *inv_per_cta = fill(g.MH, g.MW, row_cap);
    *inv_smem = ((size_t)2 * *inv_per_cta * g.MW + staged_twiddles(g.MW)) * sizeof(float2);
}

cudaError_t batched_fft_rows(const FftRowsArgs* a, BatchGrid g, int deposit_mode, size_t smem,
                             const float2* twiddles, cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    if (deposit_mode == P3M_DEPOSIT_I64)
        fft_rows_forward_batched_kernel<long long><<<g.blocks, 256, smem, s>>>(a, g.first, g.sims,
                                                                               twiddles);
    else
        fft_rows_forward_batched_kernel<uint32_t><<<g.blocks, 256, smem, s>>>(a, g.first, g.sims,
                                                                              twiddles);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t batched_fft_columns(const FftColumnsArgs* a, BatchGrid g, size_t smem,
                                const float2* twiddles, cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    fft_columns_batched_kernel<<<g.blocks, 256, smem, s>>>(a, g.first, g.sims, twiddles);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t batched_fft_inverse(const FftInverseArgs* a, BatchGrid g, size_t smem,
                                const float2* twiddles, cudaStream_t s) {
    if (g.blocks <= 0) return cudaSuccess;
    fft_rows_inverse_batched_kernel<<<g.blocks, 256, smem, s>>>(a, g.first, g.sims, twiddles);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fft_forward_columns(float2* half, GridShape g, const float2* twiddles,
                                       cudaStream_t stream) {
    int G, threads;
    column_shape(g.MW, g.MH, 2, &G, &threads, g.fft_lines);
    const int SW = g.MW / 2 + 1;
    const int blocks = (SW + G - 1) / G;
    const size_t smem = (size_t)2 * G * g.MH * sizeof(float2);
    fft_columns_forward_kernel<<<blocks, threads, smem, stream>>>(half, g.MW, g.MH, G, twiddles);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fft_inverse_rows(const float4* cols, GridShape g, const float2* twiddles,
                                    float2* force, cudaStream_t stream) {
    int rows_per_cta, threads;
    line_shape(g.MH, g.MW, g.MW >= 4096 ? 1 : 4096 / g.MW, &rows_per_cta, &threads, g.fft_lines);
    const int blocks = (g.MH + rows_per_cta - 1) / rows_per_cta;
    const size_t smem = ((size_t)2 * rows_per_cta * g.MW + staged_twiddles(g.MW)) * sizeof(float2);
    launch_chained(fft_rows_inverse_kernel, blocks, threads, smem, stream, cols, g.MW, g.MH, rows_per_cta,
                                                           twiddles, force);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_density_spectrum_f64(const void* density, int deposit_mode, double inv_scale,
                                        GridShape g, double2* z, cudaStream_t stream) {
    const long long M = (long long)g.MW * g.MH;
    density_f64_kernel<<<(int)((M + 255) / 256), 256, 0, stream>>>(
        density, deposit_mode == P3M_DEPOSIT_I64 ? 1 : 0, inv_scale, M, z);
    fft64_line_kernel<<<g.MH, 256, (size_t)g.MW * sizeof(double2), stream>>>(z, g.MW, g.MH, 0);
    fft64_line_kernel<<<g.MW, 256, (size_t)g.MH * sizeof(double2), stream>>>(z, g.MW, g.MH, 1);
    count_launches(3);
    return cudaGetLastError();
}

cudaError_t build_green(GridShape g, GreenParams p, double2* work, float2* green,
                        cudaStream_t stream) {
    const long long M = (long long)g.MW * g.MH;
    green_real_kernel<<<(int)((M + 255) / 256), 256, 0, stream>>>(
        work, g.MW, g.MH, g.W, g.H, (double)p.aspect, (double)p.gravity, (double)p.sigma_cells);
    fft64_line_kernel<<<g.MH, 256, (size_t)g.MW * sizeof(double2), stream>>>(work, g.MW, g.MH, 0);
    fft64_line_kernel<<<g.MW, 256, (size_t)g.MH * sizeof(double2), stream>>>(work, g.MW, g.MH, 1);
    const long long SWH = (long long)(g.MW / 2 + 1) * g.MH;
    green_final_kernel<<<(int)((SWH + 255) / 256), 256, 0, stream>>>(
        work, g.MW, g.MH, (double)p.window_floor, green);
    (void)ilog2_host;
    count_launches(4);
    return cudaGetLastError();
}

#endif  // !P3M_COHERENT_BODIES
}  // namespace p3m
